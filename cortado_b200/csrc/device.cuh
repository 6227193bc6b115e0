// Device building blocks of the B200 Cortado pipeline (sm_100a).
//
// Work unit: one 16 KiB chunk (4096 32-bit words) per 128-thread CTA, the
// reference's format constant CS (include/consts.h:43).  Two register layouts
// are used:
//   * group layout   -- thread g holds the 32 consecutive words 32g..32g+31;
//                       quantizers, DIFFMS and the BIT_4 transpose run here
//                       without any cross-thread traffic;
//   * segment layout -- thread t holds the 32 consecutive words 32t..32t+31
//                       of the BIT_4 output (128 bytes of one bit plane for a
//                       full chunk); zero elimination, repetition elimination
//                       and compaction run here, with one block scan.
// A 16 KiB shared-memory "plane buffer" (128-byte rows, 16-byte units XOR-
// swizzled by row, the same pattern TMA's 128B swizzle writes) moves words
// between the layouts without bank conflicts.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cortado {

constexpr int CS = 16384;   // chunk bytes (format constant)
constexpr int CW = CS / 4;  // chunk words
constexpr int NT = 128;     // threads per CTA
constexpr int HDR = 16;     // stream header bytes

// Device-latched status codes (same values as cortado_status).
enum : uint32_t {
  DST_OK = 0,
  DST_EB_TOO_SMALL = 1,
  DST_EB_TOO_LARGE = 2,
  DST_CORRUPT = 3,
  DST_SIZE_MISMATCH = 4,
  DST_TIMEOUT = 5,
  DST_CAPACITY = 10,
};

// Quantizer parameters derived from an error bound's biased exponent
// (include/d_server_encode.h:150-158).
struct Quant {
  int eb_e, thr_e, offs;
};

__host__ __device__ inline Quant make_quant(int eb_e) {
  Quant q;
  q.eb_e = eb_e;
  q.thr_e = eb_e + 24;
  q.offs = (q.thr_e << 23) - (1 << 23);
  return q;
}

// Per-launch bookkeeping shared by all CTAs (lives in the context workspace).
// The launch epoch lives in device memory (read by every CTA at start,
// advanced by the last CTA to finish), so launches captured in a CUDA graph
// get a fresh epoch on every replay.
struct Sync {
  unsigned long long* flags;  // lookback words, one per chunk (encoders)
  unsigned long long* offs;   // input payload offsets, one per chunk (decoders, re-encoders), or null
  long long flags_cap;        // words in flags and in offs (cleared when the epoch wraps)
  unsigned int* counter;      // [0] chunk queue, [1] CTAs finished, [6] helper ticket
  unsigned int* status;       // first error latched
  unsigned int* epoch;        // 0..65535, tags this launch's lookback words
  unsigned long long timeout_ns;
  int resolver;               // encoders: the helper CTA resolves lookback prefixes ahead of the flushes
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t shr_clamp(uint32_t x, uint32_t s) {
  uint32_t r;
  asm("shr.b32 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(s));  // s >= 32 gives 0
  return r;
}
__device__ __forceinline__ uint32_t shl_clamp(uint32_t x, uint32_t s) {
  uint32_t r;
  asm("shl.b32 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(s));
  return r;
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Plain arrival (no transaction bytes): release semantics, so the arriving
// thread's earlier shared-memory writes are visible to the waiters.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Waits for the phase with the given parity to complete; gives up (returns
// false) after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long limit_ns) {
  const uint32_t a = smem_u32(bar);
  uint32_t done = 0;
  unsigned long long t0 = 0;
  for (int it = 0;; ++it) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (it == 0) t0 = globaltimer();
    else if ((it & 63) == 0 && globaltimer() - t0 > limit_ns) return false;
  }
}
// 2-D tiled TMA load of a 32x128 uint32 box (one chunk, 128 rows of 128 B).
__device__ __forceinline__ void tma_load_rows(void* dst, const CUtensorMap* map, int row, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_rows(const CUtensorMap* map, int row, const void* src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(0), "r"(row), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// 1-D bulk copy global -> shared (16-byte aligned addresses and size).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// L2 prefetch of `bytes` (a multiple of 16) at a 16-byte-aligned address.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// 16 bytes from global to shared memory without a register round trip
// (the thread's own copies complete at async_wait_all); both addresses
// 16-byte aligned.
__device__ __forceinline__ void async_copy16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---------------------------------------------------------------- status
__device__ __forceinline__ void latch(unsigned int* status, unsigned int code) {
  atomicCAS(status, 0u, code);
}

// ---------------------------------------------------------------- quantizers
// Server quantizer (truncation), include/components/d_SQ_IABS_4.h:62-76.
// Values below the bound's exponent give shift >= 25, which the clamping
// shift turns into 0, so no separate test is needed.
__device__ __forceinline__ uint32_t sq_enc(uint32_t v, const Quant& q) {
  const uint32_t a = v & 0x7fffffffu;
  const int ve = (int)(a >> 23);
  const uint32_t mant = (v & 0x7fffffu) | 0x800000u;
  const uint32_t lossy = shr_clamp(mant, (uint32_t)(q.thr_e - ve));
  const uint32_t enc = (ve >= q.thr_e) ? a - (uint32_t)q.offs : lossy;
  const uint32_t s = (uint32_t)((int32_t)v >> 31);
  return (enc ^ s) - s;
}
// Client quantizer (round half away from zero), d_CQ_IABS_4.h:62-77.
__device__ __forceinline__ uint32_t cq_enc(uint32_t v, const Quant& q) {
  const uint32_t a = v & 0x7fffffffu;
  const int ve = (int)(a >> 23);
  const uint32_t sh = (uint32_t)(q.thr_e - ve);
  const uint32_t mant = (v & 0x7fffffu) | 0x800000u;
  const uint32_t lossy = shr_clamp(mant + shl_clamp(1u, sh - 1u), sh);
  const uint32_t enc = (ve >= q.thr_e) ? a - (uint32_t)q.offs : lossy;
  const uint32_t s = (uint32_t)((int32_t)v >> 31);
  return (enc ^ s) - s;
}
// Dequantizer shared by server and client bins, d_SQ_IABS_4.h:90-107.
__device__ __forceinline__ uint32_t iq_dec(uint32_t enc, const Quant& q) {
  const uint32_t neg = (uint32_t)((int32_t)enc >> 31);
  const uint32_t a = (enc ^ neg) - neg;
  const int sh = __clz(a) - 8;
  const uint32_t lossy = ((a << (sh & 31)) & 0x7fffffu) | ((uint32_t)(q.thr_e - sh) << 23);
  uint32_t dec = (a >= 0x800000u) ? a + (uint32_t)q.offs : lossy;
  dec |= enc & 0x80000000u;
  return enc ? dec : 0u;
}

// Float forms for lossy words.  A float below the bound's lossless threshold
// (|x| < 2^(thr_e - 127)) has SQ bin trunc(x * 2^(126 - eb_e)) and CQ bin
// x * 2^(126 - eb_e) rounded half away from zero; a bin below 2^23 in
// magnitude dequantizes to bin * 2^(eb_e - 126).  The scaling by a power of
// two is exact and |x| * scale < 2^23, so one multiply (or fused multiply-add
// with +-0.5) and a truncating conversion give the integer formulas' results;
// floats below 2^(eb_e - 127) have CQ bin 0 (their shift is 25 or more, and
// there the +0.5 could round the sum up to 1).  They run on the FMA and
// conversion units instead of the integer ALU.
struct FastQ {
  float sc;           // 2^(126 - eb_e)
  float dsc;          // 2^(eb_e - 126)
  uint32_t thr_bits;  // lossless threshold, as float bits (thr_e << 23)
  uint32_t lo_bits;   // 2^(eb_e - 127), as float bits
};
__device__ __forceinline__ FastQ make_fastq(int eb_e) {
  FastQ f;
  f.sc = __uint_as_float((uint32_t)(253 - eb_e) << 23);
  f.dsc = __uint_as_float((uint32_t)(eb_e + 1) << 23);
  f.thr_bits = (uint32_t)(eb_e + 24) << 23;
  f.lo_bits = (uint32_t)eb_e << 23;
  return f;
}
__device__ __forceinline__ uint32_t sq_fast(uint32_t v, const FastQ& f) {
  return (uint32_t)__float2int_rz(__fmul_rn(__uint_as_float(v), f.sc));
}
__device__ __forceinline__ uint32_t cq_fast(uint32_t v, const FastQ& f) {
  const uint32_t r =
      (uint32_t)__float2int_rz(__fmaf_rn(__uint_as_float(v), f.sc, __uint_as_float((v & 0x80000000u) | 0x3f000000u)));
  return (v & 0x7fffffffu) < f.lo_bits ? 0u : r;
}
__device__ __forceinline__ uint32_t iq_fast(uint32_t enc, const FastQ& f) {
  return __float_as_uint(__fmul_rn(__int2float_rn((int)enc), f.dsc));
}

// Per-word forms for warps that hold lossless words.  A lossless word (|x| at
// or above the threshold, inf and NaN included) has SQ and CQ bin
// +-(|x| - offs) (the exponent branch of d_SQ_IABS_4.h:62-76 and
// d_CQ_IABS_4.h:62-77), and a bin of magnitude 2^23 or more dequantizes to
// |b| + offs with b's sign bit (d_SQ_IABS_4.h:90-107); every other word takes
// the float form.  Inline selects, so no call keeps a register array live.
__device__ __forceinline__ uint32_t lossless_bin(uint32_t v, const Quant& q) {
  const uint32_t s = (uint32_t)((int32_t)v >> 31);
  return (((v & 0x7fffffffu) - (uint32_t)q.offs) ^ s) - s;
}
__device__ __forceinline__ uint32_t sq_mixed(uint32_t v, const FastQ& f, const Quant& q) {
  return (v & 0x7fffffffu) < f.thr_bits ? sq_fast(v, f) : lossless_bin(v, q);
}
__device__ __forceinline__ uint32_t cq_mixed(uint32_t v, const FastQ& f, const Quant& q) {
  return (v & 0x7fffffffu) < f.thr_bits ? cq_fast(v, f) : lossless_bin(v, q);
}
__device__ __forceinline__ uint32_t iq_mixed(uint32_t b, const FastQ& f, const Quant& q) {
  const uint32_t neg = (uint32_t)((int32_t)b >> 31);
  const uint32_t a = (b ^ neg) - neg;
  return a < 0x800000u ? iq_fast(b, f) : ((a + (uint32_t)q.offs) | (b & 0x80000000u));
}

// ---------------------------------------------------------------- BIT_4
// The reference's BIT_4 warp butterfly (include/components/d_BIT_4.h:41-92)
// maps input word i, bit b of a 32-word group to output plane 31-b, bit 31-i:
// the MSB-first 32x32 bit transpose.  Here it is done in-thread with the
// recursive block-swap transpose (H. S. Warren, Hacker's Delight, 2nd ed.,
// sec. 7-3); the 16- and 8-bit stages are byte permutes.  The transform is an
// involution, so the decoder applies the same function.
template <int J>
__device__ __forceinline__ void swap_stage(uint32_t (&a)[32], uint32_t m) {
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const int k = (i / J) * 2 * J + (i % J);
    const uint32_t t = (a[k] ^ (a[k + J] >> J)) & m;
    a[k] ^= t;
    a[k + J] ^= t << J;
  }
}
__device__ __forceinline__ void transpose32(uint32_t (&a)[32]) {
#pragma unroll
  for (int k = 0; k < 16; k++) {
    const uint32_t x = a[k], y = a[k + 16];
    a[k] = __byte_perm(x, y, 0x3276);
    a[k + 16] = __byte_perm(x, y, 0x1054);
  }
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const int k = (i / 8) * 16 + (i % 8);
    const uint32_t x = a[k], y = a[k + 8];
    a[k] = __byte_perm(x, y, 0x3715);
    a[k + 8] = __byte_perm(x, y, 0x2604);
  }
  swap_stage<4>(a, 0x0F0F0F0Fu);
  swap_stage<2>(a, 0x33333333u);
  swap_stage<1>(a, 0x55555555u);
}

// ---------------------------------------------------------------- byte masks
// 4-bit mask of the non-zero bytes of x (bit b <-> byte b).
__device__ __forceinline__ uint32_t nz_nibble(uint32_t x) {
  const uint32_t h = (((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x) & 0x80808080u;
  return ((h >> 7) * 0x01020408u) >> 24;
}
// 8-bit mask of the non-zero nibbles of x (bit i <-> nibble i).
__device__ __forceinline__ uint32_t nz_nibbles8(uint32_t x) {
  uint32_t h = ((((x & 0x77777777u) + 0x77777777u) | x) & 0x88888888u) >> 3;
  h = (h | (h >> 3)) & 0x03030303u;
  h = (h | (h >> 6)) & 0x000f000fu;
  return (h | (h >> 12)) & 0xffu;
}
// Nibble k (0..31) of a 128-bit mask held in four words.
__device__ __forceinline__ uint32_t nibble_at(const uint32_t (&M)[4], uint32_t k) {
  const uint32_t w = (k < 16) ? ((k < 8) ? M[0] : M[1]) : ((k < 24) ? M[2] : M[3]);
  return (w >> (4 * (k & 7))) & 15u;
}
// Byte-permute selector that scatters the first popc(m) bytes of a word to
// the positions of the set bits of m and zero-fills the others.
__device__ __forceinline__ uint32_t expand_sel(uint32_t m) {
  const uint32_t s = (m | (m << 3) | (m << 6) | (m << 9)) & 0x1111u;
  const uint32_t r = s * 0x1110u;
  return (r | ((s ^ 0x1111u) << 2)) & 0xffffu;
}

// ---------------------------------------------------------------- swizzle
// Linear word index -> physical word index in a 1024-byte-aligned 16 KiB
// buffer of 128-byte rows whose 16-byte units are XOR-ed with (row % 8)
// (identical to CU_TENSOR_MAP_SWIZZLE_128B).
__device__ __forceinline__ uint32_t swz(uint32_t w) {
  const uint32_t row = w >> 5;
  return (row << 5) | ((((w >> 2) & 7u) ^ (row & 7u)) << 2) | (w & 3u);
}
// Reads / writes one 128-byte row (32 words) of a swizzled buffer.
__device__ __forceinline__ void row_load(const uint32_t* buf, int row, uint32_t (&v)[32]) {
  const uint4* r = reinterpret_cast<const uint4*>(buf + row * 32);
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const uint4 u = r[k ^ (row & 7)];
    v[4 * k] = u.x;
    v[4 * k + 1] = u.y;
    v[4 * k + 2] = u.z;
    v[4 * k + 3] = u.w;
  }
}
__device__ __forceinline__ void row_store(uint32_t* buf, int row, const uint32_t (&v)[32]) {
  uint4* r = reinterpret_cast<uint4*>(buf + row * 32);
#pragma unroll
  for (int k = 0; k < 8; k++) r[k ^ (row & 7)] = make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

// ---------------------------------------------------------------- scans
// Exclusive scan over the 128 threads of a CTA; tmp holds 4 words and must not
// be reused by another scan until a later barrier.
__device__ __forceinline__ uint32_t block_scan_excl(uint32_t v, uint32_t* tmp, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) tmp[warp] = x;
  __syncthreads();
  const uint32_t w0 = tmp[0], w1 = tmp[1], w2 = tmp[2], w3 = tmp[3];
  total = w0 + w1 + w2 + w3;
  const uint32_t pre = (warp > 0 ? w0 : 0u) + (warp > 1 ? w1 : 0u) + (warp > 2 ? w2 : 0u);
  return pre + x - v;
}
__device__ __forceinline__ uint32_t warp_scan_excl(uint32_t v, uint32_t& total) {
  const int lane = threadIdx.x & 31;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}
__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------- lookback
// Lookback word: [63:48] launch epoch, [47:46] state (1 aggregate, 2 inclusive),
// [45:0] byte count.
constexpr unsigned long long LB_AGG = 1ull << 46, LB_INC = 2ull << 46, LB_VAL = (1ull << 46) - 1;

// Decoupled lookback over the chunk sizes (the role of propagate_carry,
// include/d_compression.h:120-160).  Called by one whole warp; returns the
// exclusive prefix of compressed bytes before chunk c.  Each poll reads the
// LB_WIN nearest unaccounted predecessors (LB_PER per lane, lane l covering
// distances l*LB_PER .. l*LB_PER+LB_PER-1 from the window top).  The walk ends
// at the nearest inclusive prefix if every word nearer than it has been
// published; if the whole window holds published aggregates, they are added
// and the window moves LB_WIN chunks back; otherwise the window is read
// again.  (Wider windows were measured slower: a poll that waits for a
// predecessor re-reads the whole window, and that traffic delays everyone.)
// Every wait is bounded: on timeout, or when another CTA has already failed,
// the launch's status is set and 0 is returned.  lookback_published expects
// chunk c's own word to be published already (lookback_publish), so a caller
// can do other work in between.
constexpr int LB_PER = 1;
constexpr int LB_WIN = 32 * LB_PER;

__device__ __forceinline__ unsigned long long lookback_published(const Sync& sy, unsigned int epoch, long long c,
                                                                 unsigned int csize) {
  const int lane = threadIdx.x & 31;
  const unsigned long long tag = (unsigned long long)epoch << 48;
  if (c == 0) return 0;
  unsigned long long excl = 0;
  long long top = c - 1;
  const unsigned long long t0 = globaltimer();
  int spins = 0;
  while (true) {
    // this lane's LB_PER words, nearest first
    unsigned long long f[LB_PER];
#pragma unroll
    for (int j = 0; j < LB_PER; j++) {
      const long long idx = top - (lane * LB_PER + j);
      f[j] = (idx >= 0) ? ld_relaxed(&sy.flags[idx]) : (tag | LB_INC);
    }
    int fnr = LB_PER, finc = LB_PER;  // first word not ready / first inclusive word
    unsigned long long all = 0, upto = 0;
#pragma unroll
    for (int j = LB_PER - 1; j >= 0; j--) {
      const bool ready = ((f[j] >> 48) == epoch) && ((f[j] & (3ull << 46)) != 0);
      if (!ready) fnr = j;
      if (ready && (f[j] & LB_INC)) finc = j;
    }
#pragma unroll
    for (int j = 0; j < LB_PER; j++) {
      const unsigned long long val = f[j] & LB_VAL;
      all += val;
      if (j <= finc) upto += val;
    }
    const unsigned int nr_mask = __ballot_sync(0xffffffffu, fnr < LB_PER);
    const unsigned int inc_mask = __ballot_sync(0xffffffffu, finc < LB_PER);
    const int pn = nr_mask ? __ffs(nr_mask) - 1 : 32;
    const int pi = inc_mask ? __ffs(inc_mask) - 1 : 32;
    const int fnr_pn = __shfl_sync(0xffffffffu, fnr, pn & 31);
    const int finc_pi = __shfl_sync(0xffffffffu, finc, pi & 31);
    const bool inc_first = pi < 32 && (pi < pn || (pi == pn && finc_pi < fnr_pn));
    if (inc_first) {
      excl += warp_sum64(lane < pi ? all : (lane == pi ? upto : 0ull));
      break;
    }
    if (pn == 32) {  // every word of the window is a published aggregate
      excl += warp_sum64(all);
      top -= LB_WIN;
      continue;
    }
    if ((++spins & 15) == 0) {
      int bad = 0;
      if (lane == 0) bad = (globaltimer() - t0 > sy.timeout_ns) || (*(volatile unsigned int*)sy.status != 0);
      bad = __shfl_sync(0xffffffffu, bad, 0);
      if (bad) {
        if (lane == 0) latch(sy.status, DST_TIMEOUT);
        return 0;
      }
    }
  }
  if (lane == 0) st_relaxed(&sy.flags[c], tag | LB_INC | (excl + csize));
  return excl;
}

// Publishes chunk c's own size (one thread): the inclusive prefix for chunk 0,
// the aggregate otherwise.
__device__ __forceinline__ void lookback_publish(const Sync& sy, unsigned int epoch, long long c,
                                                 unsigned int csize) {
  st_relaxed(&sy.flags[c], ((unsigned long long)epoch << 48) | (c == 0 ? LB_INC : LB_AGG) | csize);
}

__device__ __forceinline__ unsigned long long lookback(const Sync& sy, unsigned int epoch, long long c,
                                                       unsigned int csize) {
  if ((threadIdx.x & 31) == 0) lookback_publish(sy, epoch, c, csize);
  return lookback_published(sy, epoch, c, csize);
}

// Exclusive output offset of chunk c whose size was published a while ago:
// one read of its own word, which the resolver (or the chunk's predecessors'
// walks) has usually made inclusive by then; otherwise the ordinary walk.
__device__ __forceinline__ unsigned long long lookback_resolve(const Sync& sy, unsigned int epoch, long long c,
                                                               unsigned int csize) {
  const unsigned long long f = ld_relaxed(&sy.flags[c]);
  if ((f >> 48) == epoch && (f & LB_INC)) return (f & LB_VAL) - csize;
  return lookback_published(sy, epoch, c, csize);
}

// The resolver: one warp that walks the lookback words of a launch in order
// and turns every published aggregate into an inclusive prefix (running sum
// since the last inclusive word; each stream's chunk 0 publishes an inclusive
// word, so streams of a batched launch restart the sum by themselves).  It
// reads 256 words per pass and converts the published run at the front of
// them.  It stops at the end of the words or once every other CTA of the
// launch has finished; it never latches an error (the chunks' own walks still
// bound their waits).
__device__ __forceinline__ void resolve_loop(const Sync& sy, unsigned int epoch, long long total) {
  constexpr int PER = 8;
  const int lane = threadIdx.x & 31;
  const unsigned long long tag = (unsigned long long)epoch << 48;
  long long F = 0;
  unsigned long long P = 0;  // inclusive prefix of chunk F-1
  const unsigned long long t0 = globaltimer();
  while (F < total) {
    unsigned long long f[PER];
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const long long idx = F + lane * PER + j;
      f[j] = idx < total ? ld_relaxed(&sy.flags[idx]) : 0ull;
    }
    int nr = PER;
#pragma unroll
    for (int j = PER - 1; j >= 0; j--)
      if (!(((f[j] >> 48) == epoch) && ((f[j] & (3ull << 46)) != 0))) nr = j;
    const unsigned int m = __ballot_sync(0xffffffffu, nr < PER);
    const int pl = m ? __ffs(m) - 1 : 32;
    const int R = pl < 32 ? pl * PER + __shfl_sync(0xffffffffu, nr, pl) : 32 * PER;
    if (R == 0) {
      int stop = 0;
      if (lane == 0)
        stop = (*(volatile unsigned int*)&sy.counter[1] >= gridDim.x - 1) || (globaltimer() - t0 > 4 * sy.timeout_ns);
      if (__shfl_sync(0xffffffffu, stop, 0)) return;
      __nanosleep(256);
      continue;
    }
    // lane segment: positions lane*PER .. lane*PER+PER-1 below R
    const int lim = min(PER, max(0, R - lane * PER));
    bool reset = false;
    unsigned long long sum = 0;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      if (j < lim) {
        const unsigned long long v = f[j] & LB_VAL;
        if (f[j] & LB_INC) {
          reset = true;
          sum = v;
        } else {
          sum += v;
        }
      }
    }
    // inclusive segmented scan of (reset, sum) over the lanes
    bool r_in = reset;
    unsigned long long s_in = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long s_up = __shfl_up_sync(0xffffffffu, s_in, o);
      const int r_up = __shfl_up_sync(0xffffffffu, (int)r_in, o);
      if (lane >= o && !r_in) {
        s_in += s_up;
        r_in = r_up;
      }
    }
    // exclusive carry into this lane: the previous lane's inclusive value, or P
    unsigned long long carry = __shfl_up_sync(0xffffffffu, s_in, 1);
    const int carry_r = __shfl_up_sync(0xffffffffu, (int)r_in, 1);
    if (lane == 0 || !carry_r) carry = (lane == 0 ? 0ull : carry) + P;
    unsigned long long run = carry;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      if (j < lim) {
        const unsigned long long v = f[j] & LB_VAL;
        if (f[j] & LB_INC) {
          run = v;
        } else {
          run += v;
          st_relaxed(&sy.flags[F + lane * PER + j], tag | LB_INC | run);
        }
      }
    }
    // the inclusive prefix at position R-1 (held by the lane that owns it)
    const int owner = (R - 1) / PER;
    P = __shfl_sync(0xffffffffu, run, owner);
    F += R;
  }
}

// The offset scanner: one warp that turns a stream's uint16 size table into
// the byte offset of every chunk's payload (exclusive prefix sum), tagged with
// the launch epoch and a state bit like the lookback words.  32 entries per lane per pass, so
// it runs far ahead of the CTAs that read the offsets.
__device__ __forceinline__ void scan_offsets(unsigned long long* offs, unsigned int epoch, const uint16_t* table,
                                             long long chunks) {
  constexpr int PER = 32;
  const int lane = threadIdx.x & 31;
  const unsigned long long tag = (unsigned long long)epoch << 48;
  unsigned long long run = 0;
  for (long long i = 0; i < chunks; i += 32 * PER) {
    const long long b = i + (long long)lane * PER;
    uint32_t e[PER];
    if (b + PER <= chunks) {
#pragma unroll
      for (int k = 0; k < PER / 8; k++) {
        const uint4 w = *reinterpret_cast<const uint4*>(table + b + 8 * k);
        e[8 * k + 0] = w.x & 0xffffu; e[8 * k + 1] = w.x >> 16;
        e[8 * k + 2] = w.y & 0xffffu; e[8 * k + 3] = w.y >> 16;
        e[8 * k + 4] = w.z & 0xffffu; e[8 * k + 5] = w.z >> 16;
        e[8 * k + 6] = w.w & 0xffffu; e[8 * k + 7] = w.w >> 16;
      }
    } else {
#pragma unroll
      for (int j = 0; j < PER; j++) e[j] = (b + j < chunks) ? table[b + j] : 0u;
    }
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < PER; j++) sum += e[j];
    uint32_t total;
    const uint32_t base = warp_scan_excl(sum, total);
    unsigned long long o = run + base;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      if (b + j < chunks) offs[b + j] = tag | LB_INC | o;  // the state bit: a zeroed word is never valid
      o += e[j];
    }
    run += total;
  }
}

// Offset of chunk c's payload from the scanner's word (waits, bounded, until
// the word carries this launch's epoch; on timeout latches the status and
// returns 0).
__device__ __forceinline__ unsigned long long wait_offset(const Sync& sy, unsigned int epoch, long long c) {
  const unsigned long long t0 = globaltimer();
  for (int it = 0;; ++it) {
    const unsigned long long v = ld_relaxed(&sy.offs[c]);
    if ((v >> 48) == epoch && (v & LB_INC)) return v & LB_VAL;
    if ((it & 15) == 15) {
      if (globaltimer() - t0 > sy.timeout_ns || *(volatile unsigned int*)sy.status != 0) {
        latch(sy.status, DST_TIMEOUT);
        return 0;
      }
      __nanosleep(128);
    }
  }
}

}  // namespace cortado
