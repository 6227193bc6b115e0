/*
 * cortado_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's per-chunk encode/decode path, used
 * as the parity oracle for the CUDA kernels.  Only tests/, the smoke() entry
 * point and bench.py's CPU-baseline legs may load this library; the product
 * library (libcortado.so) never links or calls it.
 *
 * Pinning: the streams and decoded floats this file produces are checked
 * byte-for-byte against outputs of the reference's own CLI binaries (built
 * from the reference sources by oracle/ref.mk, run on a B200) in
 * tests/golden/.  Header bytes 12..15 are masked in that comparison because
 * the reference never writes them (include/d_server_encode.h:134-138).
 *
 * Each routine follows the DEVICE code of the reference (not its unused
 * host-side h_RZE.h, whose capacity checks differ):
 *   quantizers  include/components/d_SQ_IABS_4.h:51-109,
 *               include/components/d_CQ_IABS_4.h:51-110,
 *               include/preprocessors/include/IABS_f32.h:44-113
 *   residual    include/components/d_RESI_4.h:57-94
 *   DIFFMS      include/components/include/d_DIFFMS.h:44-102
 *   BIT_4       include/components/d_BIT_4.h:41-144 (butterfly emulated lane by lane)
 *   RZE_1       include/components/include/d_RZE.h:48-206,
 *               include/components/include/d_zero_elimination.h:45-113, 810-869,
 *               include/components/include/d_repetition_elimination.h:121-185,
 *               283-409, 574-616, 675-742
 *   kernels     include/d_server_encode.h:51-260, include/d_s2c.h:51-224,
 *               include/d_client_encode.h:173-266, include/d_residual_encode.h:51-354
 *   verifier    include/verifiers/MAXABS_f32.h:40-72
 *
 * Defined behaviour where the reference is undefined (the CUDA product
 * follows the same definitions):
 *   - input sizes must be a multiple of 4 bytes (the reference's quantizers
 *     leave trailing bytes of a non-multiple-of-4 chunk as stale shared memory);
 *   - header bytes 12..15 are written as 0;
 *   - dequantizing the int32 bin INT_MIN treats its magnitude as 2^31
 *     (the reference negates it with signed overflow);
 *   - corrupt streams return CORTADO_ORACLE_CORRUPT instead of trapping.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CS 16384
#define HDR 16

enum {
  ORA_OK = 0,
  ORA_EB_TOO_SMALL = 1,
  ORA_EB_TOO_LARGE = 2,
  ORA_CORRUPT = 3,
  ORA_SIZE_MISMATCH = 4,
  ORA_INVALID_ARG = 7,
  ORA_CAPACITY = 10,
};

typedef struct { int eb_e, thr_e, offs; } qp_t;

/* Error-bound exponent plumbing: include/d_server_encode.h:150-158,
 * include/d_s2c.h:208-214, include/d_residual_encode.h:211-223. */
int ora_eb_params(float eb, int* eb_e, int* thr_e, int* offs)
{
  if (eb < FLT_MIN) return ORA_EB_TOO_SMALL;
  uint32_t bits;
  memcpy(&bits, &eb, 4);
  const int e = (int)((bits >> 23) & 0xff);
  const int t = e + 24;
  if (t >= 255) return ORA_EB_TOO_LARGE;
  *eb_e = e;
  *thr_e = t;
  *offs = (t << 23) - (1 << 23);
  return ORA_OK;
}

static qp_t qp_from_exp(int eb_e)
{
  qp_t q;
  q.eb_e = eb_e;
  q.thr_e = eb_e + 24;
  q.offs = (q.thr_e << 23) - (1 << 23);
  return q;
}

/* d_SQ_IABS_4.h:62-76 (server quantizer: truncation toward zero) */
static int32_t sq_enc(uint32_t val, qp_t q)
{
  const int32_t a = (int32_t)(val & 0x7fffffffu);
  const int ve = a >> 23;
  int32_t enc = 0;
  if (ve >= q.thr_e) {
    enc = a - q.offs;
  } else if (ve >= q.eb_e) {
    int32_t mant = (int32_t)((val & 0x7fffffu) | (1u << 23));
    enc = mant >> (q.thr_e - ve);
  }
  if (val >> 31) enc = -enc;
  return enc;
}

/* d_CQ_IABS_4.h:62-77 and IABS_f32.h:72-90 (client quantizer: rounding) */
static int32_t cq_enc(uint32_t val, qp_t q)
{
  const int32_t a = (int32_t)(val & 0x7fffffffu);
  const int ve = a >> 23;
  int32_t enc = 0;
  if (ve >= q.thr_e) {
    enc = a - q.offs;
  } else if (ve >= q.eb_e) {
    const int sh = q.thr_e - ve;
    int32_t mant = (int32_t)((val & 0x7fffffu) | (1u << 23));
    mant += 1 << (sh - 1);
    enc = mant >> sh;
  }
  if (val >> 31) enc = -enc;
  return enc;
}

/* d_SQ_IABS_4.h:90-107, d_CQ_IABS_4.h:91-108, IABS_f32.h:46-62, 93-113
 * (server and client dequantizers are identical). */
static uint32_t iq_dec(int32_t enc, qp_t q)
{
  uint32_t dec = 0;
  if (enc != 0) {
    const uint32_t a = (enc < 0) ? 0u - (uint32_t)enc : (uint32_t)enc;
    if (a >= (1u << 23)) {
      dec = a + (uint32_t)q.offs;
    } else {
      const int sh = __builtin_clz(a) - 8;
      dec = a << sh;
      dec &= 0x7fffffu;
      dec |= (uint32_t)(q.thr_e - sh) << 23;
    }
    dec |= (uint32_t)enc & 0x80000000u;
  }
  return dec;
}

/* ---------- DIFFMS (d_DIFFMS.h:44-102) ---------- */
static void diffms(const uint8_t* in, uint8_t* out, int csize)
{
  const int size = csize / 4;
  uint32_t prev = 0;
  for (int i = 0; i < size; i++) {
    uint32_t v;
    memcpy(&v, in + 4 * i, 4);
    const uint32_t d = v - prev;
    const uint32_t z = (d << 1) ^ (uint32_t)((int32_t)d >> 31);
    memcpy(out + 4 * i, &z, 4);
    prev = v;
  }
  for (int i = size * 4; i < csize; i++) out[i] = in[i];
}

static void idiffms(const uint8_t* in, uint8_t* out, int csize)
{
  const int size = csize / 4;
  uint32_t sum = 0;
  for (int i = 0; i < size; i++) {
    uint32_t z;
    memcpy(&z, in + 4 * i, 4);
    const uint32_t d = (z >> 1) ^ (uint32_t)((int32_t)(z << 31) >> 31);
    sum += d;
    memcpy(out + 4 * i, &sum, 4);
  }
  for (int i = size * 4; i < csize; i++) out[i] = in[i];
}

/* ---------- BIT_4 (d_BIT_4.h:41-144): the 32-lane butterfly, emulated ---------- */
static uint32_t byte_perm(uint32_t x, uint32_t y, uint32_t s)
{
  uint8_t b[8];
  for (int i = 0; i < 4; i++) { b[i] = (uint8_t)(x >> (8 * i)); b[4 + i] = (uint8_t)(y >> (8 * i)); }
  uint32_t r = 0;
  for (int i = 0; i < 4; i++) r |= (uint32_t)b[(s >> (4 * i)) & 7] << (8 * i);
  return r;
}

static void butterfly(uint32_t a[32])
{
  uint32_t q[32];
  for (int l = 0; l < 32; l++) q[l] = a[l ^ 16];
  for (int l = 0; l < 32; l++)
    a[l] = ((l & 16) == 0) ? byte_perm(a[l], q[l], (3 << 12) | (2 << 8) | (7 << 4) | 6)
                           : byte_perm(a[l], q[l], (5 << 12) | (4 << 8) | (1 << 4) | 0);
  for (int l = 0; l < 32; l++) q[l] = a[l ^ 8];
  for (int l = 0; l < 32; l++)
    a[l] = ((l & 8) == 0) ? byte_perm(a[l], q[l], (3 << 12) | (7 << 8) | (1 << 4) | 5)
                          : byte_perm(a[l], q[l], (6 << 12) | (2 << 8) | (4 << 4) | 0);
  static const uint32_t masks[3] = {0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
  static const int shifts[3] = {4, 2, 1};
  for (int st = 0; st < 3; st++) {
    const int k = shifts[st];
    const uint32_t m = masks[st];
    for (int l = 0; l < 32; l++) q[l] = a[l ^ k];
    for (int l = 0; l < 32; l++) {
      if ((l & k) == 0) a[l] = (a[l] & ~m) | ((q[l] >> k) & m);
      else a[l] = ((q[l] << k) & ~m) | (a[l] & m);
    }
  }
}

static void bit4(const uint8_t* in, uint8_t* out, int csize)
{
  const int extra = csize % 128;
  const int size = (csize - extra) / 4;
  const int G = size / 32;
  for (int g = 0; g < G; g++) {
    uint32_t a[32];
    memcpy(a, in + 128 * g, 128);
    butterfly(a);
    for (int s = 0; s < 32; s++) memcpy(out + 4 * (g + s * G), &a[s], 4);
  }
  for (int i = csize - extra; i < csize; i++) out[i] = in[i];
}

static void ibit4(const uint8_t* in, uint8_t* out, int csize)
{
  const int extra = csize % 128;
  const int size = (csize - extra) / 4;
  const int G = size / 32;
  for (int g = 0; g < G; g++) {
    uint32_t a[32];
    for (int s = 0; s < 32; s++) memcpy(&a[s], in + 4 * (g + s * G), 4);
    butterfly(a);
    memcpy(out + 128 * g, a, 128);
  }
  for (int i = csize - extra; i < csize; i++) out[i] = in[i];
}

/* ---------- RZE_1 (d_RZE.h:48-206 with T = byte) ---------- */
/* One repetition-elimination level on n bytes (d_REencode*, check = true):
 * keep byte i iff it differs from byte i-1 (byte -1 is 0); bit i of bm_out
 * marks a kept byte.  Fails without writing when more than cap bytes are kept
 * (d_repetition_elimination.h:166-167, 394-395). */
static int re_level(const uint8_t* in, int n, uint8_t* out, int* wpos, int cap, uint8_t* bm_out)
{
  int cnt = 0;
  for (int i = 0; i < n; i++) cnt += (in[i] != (i ? in[i - 1] : 0));
  if (cnt > cap) return 0;
  memset(bm_out, 0, (size_t)n / 8);
  for (int i = 0; i < n; i++) {
    if (in[i] != (i ? in[i - 1] : 0)) {
      bm_out[i / 8] |= (uint8_t)(1u << (i % 8));
      out[(*wpos)++] = in[i];
    }
  }
  return 1;
}

static int rze(const uint8_t* in, int csize, uint8_t* out, int* new_csize)
{
  const int avail = CS - 2;
  uint8_t bm[2048 + 256 + 32 + 4];
  memset(bm, 0, sizeof(bm));
  int wpos = 0;
  for (int k = 0; k < csize; k++) {  /* d_ZEencodebyteshort (d_zero_elimination.h:45-113) */
    if (in[k]) {
      bm[k / 8] |= (uint8_t)(1u << (k % 8));
      out[wpos++] = in[k];
    }
  }
  if (wpos >= avail) return 0;                                      /* d_RZE.h:72 */
  if (wpos != 0) {
    if (!re_level(&bm[0], 2048, out, &wpos, avail - wpos, &bm[2048])) return 0;          /* :81 */
    if (!re_level(&bm[2048], 256, out, &wpos, avail - wpos, &bm[2304])) return 0;        /* :88 */
    if (!re_level(&bm[2304], 32, out, &wpos, avail - wpos, &bm[2336])) return 0;         /* :96 */
    if (wpos >= avail - 4) return 0;                                                      /* :104 */
    memcpy(out + wpos, &bm[2336], 4);
    wpos += 4;
  }
  out[wpos] = (uint8_t)csize;
  out[wpos + 1] = (uint8_t)(csize >> 8);
  *new_csize = wpos + 2;
  return 1;
}

/* d_REdecode*: byte i = last kept byte at or before i (0 if none). */
static int re_decode(int n, const uint8_t* data, int avail, const uint8_t* bm, uint8_t* out)
{
  int pos = 0;
  uint8_t val = 0;
  for (int i = 0; i < n; i++) {
    if ((bm[i / 8] >> (i % 8)) & 1) {
      if (pos >= avail) return 0;
      val = data[pos++];
    }
    out[i] = val;
  }
  return 1;
}

static int popc_bytes(const uint8_t* b, int n)
{
  int c = 0;
  for (int i = 0; i < n; i++) c += __builtin_popcount(b[i]);
  return c;
}

/* d_iRZE (d_RZE.h:127-206); returns 0 on a malformed chunk. */
static int irze(const uint8_t* in, int csize_in, uint8_t* out, int* csize_out)
{
  if (csize_in < 2) return 0;
  int rpos = csize_in;
  int csize = (int)in[--rpos] << 8;
  csize |= in[--rpos];
  if (csize > CS) return 0;
  *csize_out = csize;
  if (rpos == 0) {
    memset(out, 0, (size_t)csize);
    return 1;
  }
  uint8_t bm[2048 + 256 + 32 + 4];
  rpos -= 4;
  if (rpos < 0) return 0;
  memcpy(&bm[2336], in + rpos, 4);
  int c = popc_bytes(&bm[2336], 4);
  rpos -= c;
  if (rpos < 0) return 0;
  if (!re_decode(32, in + rpos, c, &bm[2336], &bm[2304])) return 0;
  c = popc_bytes(&bm[2304], 32);
  rpos -= c;
  if (rpos < 0) return 0;
  if (!re_decode(256, in + rpos, c, &bm[2304], &bm[2048])) return 0;
  c = popc_bytes(&bm[2048], 256);
  rpos -= c;
  if (rpos < 0) return 0;
  if (!re_decode(2048, in + rpos, c, &bm[2048], &bm[0])) return 0;
  /* d_ZEdecode byte path (d_zero_elimination.h:846-868): non-zero bytes from in[0..) */
  int pos = 0;
  for (int k = 0; k < csize; k++) {
    if ((bm[k / 8] >> (k % 8)) & 1) {
      if (pos >= rpos) return 0;
      out[k] = in[pos++];
    } else {
      out[k] = 0;
    }
  }
  /* bits beyond csize must be clear and every data byte consumed */
  for (int k = csize; k < CS; k++)
    if ((bm[k / 8] >> (k % 8)) & 1) return 0;
  if (pos != rpos) return 0;
  return 1;
}

/* ---------- per-chunk pipelines ---------- */
enum { MODE_STORE = 0, MODE_S2C = 1, MODE_RESI = 2 };

/* Shared encode tail: DIFFMS -> BIT_4 -> RZE_1 on words[0..osize) with the
 * raw fallback of d_server_encode.h:112-126 / d_s2c.h:164-183 /
 * d_residual_encode.h:165-184: a chunk whose result is not smaller than the
 * input is stored as the pre-pipeline bytes `raw`. */
static int encode_words(const uint8_t* words, int osize, const uint8_t* raw, uint8_t* out)
{
  uint8_t b1[CS + 8], b2[CS + 8];
  diffms(words, b1, osize);
  bit4(b1, b2, osize);
  int csize = 0;
  const int good = rze(b2, osize, out, &csize);
  if (!good || csize >= osize) {
    memcpy(out, raw, (size_t)osize);
    csize = osize;
  }
  return csize;
}

/* Decode a compressed (csize < osize) chunk to its pre-pipeline words. */
static int decode_words(const uint8_t* payload, int csize, int osize, uint8_t* words)
{
  uint8_t b1[CS + 8], b2[CS + 8];
  int c2 = 0;
  if (!irze(payload, csize, b1, &c2)) return 0;
  if (c2 != osize) return 0;
  ibit4(b1, b2, osize);
  idiffms(b2, words, osize);
  return 1;
}

/* ---------- stream helpers ---------- */
static int64_t nchunks(int64_t n) { return (n + CS - 1) / CS; }

int64_t ora_max_stream_bytes(int64_t n) { return HDR + 2 * nchunks(n) + nchunks(n) * (int64_t)CS; }

static void write_header(uint8_t* out, int64_t n, int eb_e)
{
  memcpy(out, &n, 8);
  int32_t e = eb_e, z = 0;
  memcpy(out + 8, &e, 4);
  memcpy(out + 12, &z, 4);
}

typedef struct {
  int64_t n, chunks;
  int eb_e;
  const uint16_t* sizes_unaligned;
  const uint8_t* data;
  int64_t* offs; /* chunks + 1 */
} parsed_t;

static uint16_t rd16(const uint8_t* p) { return (uint16_t)(p[0] | (p[1] << 8)); }

static int parse_stream(const uint8_t* s, int64_t bytes, parsed_t* p)
{
  if (bytes < HDR) return ORA_CORRUPT;
  memcpy(&p->n, s, 8);
  int32_t e;
  memcpy(&e, s + 8, 4);
  p->eb_e = e;
  if (p->n < 0 || (p->n & 3)) return ORA_CORRUPT;
  if (e < 1 || e > 230) return ORA_CORRUPT;
  p->chunks = nchunks(p->n);
  if (bytes < HDR + 2 * p->chunks) return ORA_CORRUPT;
  p->data = s + HDR + 2 * p->chunks;
  p->offs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(p->chunks + 1));
  p->offs[0] = 0;
  for (int64_t c = 0; c < p->chunks; c++) {
    const int cs = rd16(s + HDR + 2 * c);
    const int os = (int)((p->n - c * CS) < CS ? (p->n - c * CS) : CS);
    if (cs > os || cs < 1) { free(p->offs); return ORA_CORRUPT; }
    p->offs[c + 1] = p->offs[c] + cs;
  }
  if (HDR + 2 * p->chunks + p->offs[p->chunks] > bytes) { free(p->offs); return ORA_CORRUPT; }
  p->sizes_unaligned = (const uint16_t*)(s + HDR);
  return ORA_OK;
}

/* Assemble per-chunk results (two-pass: chunks encoded independently, then
 * an exclusive scan of their sizes places them; the reference does the same
 * with a decoupled lookback, d_compression.h:120-160). */
static int64_t assemble(uint8_t* out, int64_t n, int eb_e, int64_t chunks, uint8_t* tmp, const int* csz, int nthreads)
{
  write_header(out, n, eb_e);
  int64_t* offs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(chunks + 1));
  offs[0] = 0;
  for (int64_t c = 0; c < chunks; c++) {
    out[HDR + 2 * c] = (uint8_t)csz[c];
    out[HDR + 2 * c + 1] = (uint8_t)(csz[c] >> 8);
    offs[c + 1] = offs[c] + csz[c];
  }
  uint8_t* data = out + HDR + 2 * chunks;
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t c = 0; c < chunks; c++) memcpy(data + offs[c], tmp + c * (int64_t)CS, (size_t)csz[c]);
  const int64_t total = HDR + 2 * chunks + offs[chunks];
  free(offs);
  return total;
}

static int osize_of(int64_t n, int64_t c) { return (int)((n - c * CS) < CS ? (n - c * CS) : CS); }

/* ---------- operations ---------- */

/* store: d_server_encode (d_server_encode.h:146-166) -- eb_abs is the client
 * bound; the stored bins use eb_abs/2. */
int ora_store_encode(const uint8_t* in, int64_t n, float eb_abs, uint8_t* out, int64_t cap, int64_t* outsize, int nthreads)
{
  if (n < 0 || (n & 3)) return ORA_INVALID_ARG;
  int eb_e, thr_e, offs;
  const int st = ora_eb_params(eb_abs / 2, &eb_e, &thr_e, &offs);
  if (st) return st;
  const int64_t chunks = nchunks(n);
  if (cap < ora_max_stream_bytes(n)) return ORA_CAPACITY;
  const qp_t q = qp_from_exp(eb_e);
  uint8_t* tmp = (uint8_t*)malloc((size_t)(chunks ? chunks : 1) * CS);
  int* csz = (int*)malloc(sizeof(int) * (size_t)(chunks ? chunks : 1));
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
  for (int64_t c = 0; c < chunks; c++) {
    const int os = osize_of(n, c);
    const uint8_t* src = in + c * (int64_t)CS;
    uint8_t w[CS + 8];
    for (int i = 0; i < os / 4; i++) {
      uint32_t v;
      memcpy(&v, src + 4 * i, 4);
      const uint32_t e = (uint32_t)sq_enc(v, q);
      memcpy(w + 4 * i, &e, 4);
    }
    csz[c] = encode_words(w, os, src, tmp + c * (int64_t)CS);
  }
  *outsize = assemble(out, n, eb_e, chunks, tmp, csz, nthreads);
  free(tmp);
  free(csz);
  return ORA_OK;
}

/* Decoders.  kind 0: storage decode (iSQ, d_server_encode.h:169-260);
 * kind 1: init_recv (iCQ, d_client_encode.h:173-259; raw chunks are copied
 * out undequantized, as the reference does). */
static int decode_stream(const uint8_t* s, int64_t bytes, uint8_t* out, int64_t cap, int64_t* outsize, int kind, int nthreads)
{
  parsed_t p;
  int st = parse_stream(s, bytes, &p);
  if (st) return st;
  if (cap < p.n) { free(p.offs); return ORA_CAPACITY; }
  const qp_t q = qp_from_exp(p.eb_e);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(| : bad)
  for (int64_t c = 0; c < p.chunks; c++) {
    const int os = osize_of(p.n, c);
    const int cs = (int)(p.offs[c + 1] - p.offs[c]);
    uint8_t* dst = out + c * (int64_t)CS;
    if (cs == os) {
      memcpy(dst, p.data + p.offs[c], (size_t)os);
      continue;
    }
    uint8_t w[CS + 8];
    if (!decode_words(p.data + p.offs[c], cs, os, w)) { bad = 1; memset(dst, 0, (size_t)os); continue; }
    for (int i = 0; i < os / 4; i++) {
      int32_t e;
      memcpy(&e, w + 4 * i, 4);
      const uint32_t d = iq_dec(e, q);
      memcpy(dst + 4 * i, &d, 4);
    }
  }
  (void)kind;
  *outsize = p.n;
  free(p.offs);
  return bad ? ORA_CORRUPT : ORA_OK;
}

int ora_store_decode(const uint8_t* s, int64_t bytes, uint8_t* out, int64_t cap, int64_t* outsize, int nthreads)
{
  return decode_stream(s, bytes, out, cap, outsize, 0, nthreads);
}

int ora_init_recv(const uint8_t* s, int64_t bytes, uint8_t* out, int64_t cap, int64_t* outsize, int nthreads)
{
  return decode_stream(s, bytes, out, cap, outsize, 1, nthreads);
}

/* init_send: d_s2c_encode (d_s2c.h:51-224); resi_send: d_residual_encode
 * (d_residual_encode.h:51-230).  Both decode the stored chunk (iSQ), then
 * requantize (CQ at the request bound) or form the residual (RESI), then
 * encode; an incompressible chunk is stored as those bins / residuals. */
static int reencode(const uint8_t* s, int64_t bytes, int mode, float eb1, float eb2, uint8_t* out, int64_t cap, int64_t* outsize, int nthreads)
{
  int a_e, a_t, a_o, b_e = 0, b_t = 0, b_o = 0;
  int st = ora_eb_params(eb1, &a_e, &a_t, &a_o);
  if (st) return st;
  if (mode == MODE_RESI) {
    st = ora_eb_params(eb2, &b_e, &b_t, &b_o);
    if (st) return st;
  }
  parsed_t p;
  st = parse_stream(s, bytes, &p);
  if (st) return st;
  if (cap < ora_max_stream_bytes(p.n)) { free(p.offs); return ORA_CAPACITY; }
  const qp_t sq = qp_from_exp(p.eb_e);
  const qp_t qa = qp_from_exp(a_e);
  const qp_t qb = qp_from_exp(b_e);
  const int64_t chunks = p.chunks;
  uint8_t* tmp = (uint8_t*)malloc((size_t)(chunks ? chunks : 1) * CS);
  int* csz = (int*)malloc(sizeof(int) * (size_t)(chunks ? chunks : 1));
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(| : bad)
  for (int64_t c = 0; c < chunks; c++) {
    const int os = osize_of(p.n, c);
    const int cs = (int)(p.offs[c + 1] - p.offs[c]);
    uint8_t x[CS + 8], w[CS + 8];
    if (cs == os) {
      memcpy(x, p.data + p.offs[c], (size_t)os);
    } else {
      if (!decode_words(p.data + p.offs[c], cs, os, w)) { bad = 1; memset(w, 0, (size_t)os); }
      for (int i = 0; i < os / 4; i++) {
        int32_t e;
        memcpy(&e, w + 4 * i, 4);
        const uint32_t d = iq_dec(e, sq);
        memcpy(x + 4 * i, &d, 4);
      }
    }
    for (int i = 0; i < os / 4; i++) {
      uint32_t v;
      memcpy(&v, x + 4 * i, 4);
      uint32_t r;
      if (mode == MODE_S2C) {
        r = (uint32_t)cq_enc(v, qa);
      } else {  /* d_RESI_4.h:67-74 */
        const int32_t src = cq_enc(v, qa);
        const uint32_t src_deq = iq_dec(src, qa);
        const int32_t src_req = cq_enc(src_deq, qb);
        const int32_t dst = cq_enc(v, qb);
        r = (uint32_t)dst - (uint32_t)src_req;
      }
      memcpy(w + 4 * i, &r, 4);
    }
    csz[c] = encode_words(w, os, w, tmp + c * (int64_t)CS);
  }
  *outsize = assemble(out, p.n, mode == MODE_S2C ? a_e : b_e, chunks, tmp, csz, nthreads);
  free(tmp);
  free(csz);
  free(p.offs);
  return bad ? ORA_CORRUPT : ORA_OK;
}

int ora_init_send(const uint8_t* s, int64_t bytes, float request_eb, uint8_t* out, int64_t cap, int64_t* outsize, int nthreads)
{
  return reencode(s, bytes, MODE_S2C, request_eb, 0.0f, out, cap, outsize, nthreads);
}

int ora_resi_send(const uint8_t* s, int64_t bytes, float src_eb, float dst_eb, uint8_t* out, int64_t cap, int64_t* outsize, int nthreads)
{
  return reencode(s, bytes, MODE_RESI, src_eb, dst_eb, out, cap, outsize, nthreads);
}

/* resi_recv: d_residual_apply (d_residual_encode.h:238-354). */
int ora_resi_recv(const uint8_t* src, int64_t n, const uint8_t* s, int64_t bytes, uint8_t* out, int64_t cap, int64_t* outsize, int nthreads)
{
  parsed_t p;
  int st = parse_stream(s, bytes, &p);
  if (st) return st;
  if (p.n != n) { free(p.offs); return ORA_SIZE_MISMATCH; }
  if (cap < n) { free(p.offs); return ORA_CAPACITY; }
  const qp_t q = qp_from_exp(p.eb_e);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(| : bad)
  for (int64_t c = 0; c < p.chunks; c++) {
    const int os = osize_of(p.n, c);
    const int cs = (int)(p.offs[c + 1] - p.offs[c]);
    uint8_t r[CS + 8];
    if (cs == os) {
      memcpy(r, p.data + p.offs[c], (size_t)os);
    } else if (!decode_words(p.data + p.offs[c], cs, os, r)) {
      bad = 1;
      memset(r, 0, (size_t)os);
    }
    const uint8_t* sc = src + c * (int64_t)CS;
    uint8_t* dst = out + c * (int64_t)CS;
    for (int i = 0; i < os / 4; i++) {  /* d_RESI_4.h:88-92 */
      uint32_t v, rr;
      memcpy(&v, sc + 4 * i, 4);
      memcpy(&rr, r + 4 * i, 4);
      const int32_t req = cq_enc(v, q);
      const uint32_t d = iq_dec((int32_t)((uint32_t)req + rr), q);
      memcpy(dst + 4 * i, &d, 4);
    }
  }
  *outsize = n;
  free(p.offs);
  return bad ? ORA_CORRUPT : ORA_OK;
}

/* iCQ(CQ(x, eb)): the stand-alone client quantizer pair the reference's -v
 * paths compare decoded output against (d_client_QUANT_IABS_0_f32.h:51-143,
 * cortado_init.cu:515-534). */
int ora_client_roundtrip(const float* x, int64_t nw, float eb_abs, float* out)
{
  int e, t, o;
  const int st = ora_eb_params(eb_abs, &e, &t, &o);
  if (st) return st;
  const qp_t q = qp_from_exp(e);
  for (int64_t i = 0; i < nw; i++) {
    uint32_t v;
    memcpy(&v, &x[i], 4);
    const uint32_t d = iq_dec(cq_enc(v, q), q);
    memcpy(&out[i], &d, 4);
  }
  return ORA_OK;
}

/* MAXABS_f32 (MAXABS_f32.h:40-72): returns -1 if every value is within eb,
 * else the first violating index. */
int64_t ora_maxabs(const float* recon, const float* orig, int64_t nw, float eb)
{
  for (int64_t i = 0; i < nw; i++) {
    const float o = orig[i], r = recon[i];
    if (!isfinite(o) || !isfinite(r)) {
      if (r != o && (!isnan(o) || !isnan(r))) return i;
    } else {
      const float lower = o - eb;
      const float upper = o + eb;
      if (r < lower || r > upper || fabsf(o - r) > eb) return i;
    }
  }
  return -1;
}

/* Per-stage entry points, for unit tests of the oracle itself. */
void ora_bit4(const uint8_t* in, uint8_t* out, int csize) { bit4(in, out, csize); }
void ora_ibit4(const uint8_t* in, uint8_t* out, int csize) { ibit4(in, out, csize); }
int ora_rze(const uint8_t* in, int csize, uint8_t* out) { int c = 0; return rze(in, csize, out, &c) ? c : -1; }
int ora_irze(const uint8_t* in, int csize, uint8_t* out) { int c = 0; return irze(in, csize, out, &c) ? c : -1; }
uint32_t ora_sq(uint32_t v, int eb_e) { return (uint32_t)sq_enc(v, qp_from_exp(eb_e)); }
uint32_t ora_cq(uint32_t v, int eb_e) { return (uint32_t)cq_enc(v, qp_from_exp(eb_e)); }
uint32_t ora_iq(uint32_t v, int eb_e) { return iq_dec((int32_t)v, qp_from_exp(eb_e)); }
