/* Check of the float forms of the quantizers used for lossy words (server
 * quantizer SQ, client quantizer CQ, dequantizer iQ) against the oracle's
 * integer restatements of the reference's d_SQ_IABS_4 / d_CQ_IABS_4 /
 * d_iSQ_IABS_4, on every input: the float forms for lossy words and bins,
 * the integer shortcuts for lossless ones (the kernels' *_mixed forms).
 * Test infrastructure only: links the CPU oracle.
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off quant_fast_check.c -lm -L<oracle> -lcortado_oracle
 * Usage: quant_fast_check <eb_e> <stride>   (stride 1: every 32-bit input)
 * Prints checked and mismatching counts; exit status 1 on any mismatch. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

uint32_t ora_sq(uint32_t v, int eb_e);
uint32_t ora_cq(uint32_t v, int eb_e);
uint32_t ora_iq(uint32_t v, int eb_e);

static float f_of(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t u_of(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* the device's forms (round-toward-zero conversion, exact power-of-two scales) */
static uint32_t sq_fast(uint32_t v, float sc) { return (uint32_t)(int32_t)truncf(f_of(v) * sc); }
/* words below 2^(eb_e - 127) quantize to 0 (a shift of 25 or more); above
 * that, |x| * scale + 0.5 is exact, so the truncation rounds half away */
static uint32_t cq_fast(uint32_t v, float sc, uint32_t lo_bits) {
  if ((v & 0x7fffffffu) < lo_bits) return 0u;
  return (uint32_t)(int32_t)truncf(fmaf(f_of(v), sc, f_of((v & 0x80000000u) | 0x3f000000u)));
}
static uint32_t iq_fast(uint32_t e, float dsc) { return u_of((float)(int32_t)e * dsc); }

/* the per-word forms for any input: lossless words (and inf, NaN) take
 * +-(|x| - offs), bins of magnitude 2^23 or more |b| + offs with b's sign */
static uint32_t lossless_bin(uint32_t v, uint32_t offs) {
  const uint32_t s = (uint32_t)((int32_t)v >> 31);
  return (((v & 0x7fffffffu) - offs) ^ s) - s;
}
static uint32_t iq_mixed(uint32_t b, float dsc, uint32_t offs) {
  const uint32_t neg = (uint32_t)((int32_t)b >> 31), a = (b ^ neg) - neg;
  return a < 0x800000u ? iq_fast(b, dsc) : ((a + offs) | (b & 0x80000000u));
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const int eb_e = atoi(argv[1]);
  const long long stride = atoll(argv[2]);
  const uint32_t thr_bits = (uint32_t)(eb_e + 24) << 23;
  const float sc = f_of((uint32_t)(253 - eb_e) << 23);  /* 2^(126 - eb_e) */
  const float dsc = f_of((uint32_t)(eb_e + 1) << 23);   /* 2^(eb_e - 126) */
  const uint32_t offs = thr_bits - (1u << 23);
  long long checked = 0, bad = 0;
#pragma omp parallel for reduction(+ : checked, bad) schedule(static)
  for (long long i = 0; i < (1ll << 32); i += stride) {
    const uint32_t v = (uint32_t)i;
    const int lossy = (v & 0x7fffffffu) < thr_bits;
    const uint32_t sq = lossy ? sq_fast(v, sc) : lossless_bin(v, offs);
    const uint32_t cq = lossy ? cq_fast(v, sc, (uint32_t)eb_e << 23) : lossless_bin(v, offs);
    checked += 3;
    if (sq != ora_sq(v, eb_e)) bad++;
    if (cq != ora_cq(v, eb_e)) bad++;
    if (iq_mixed(v, dsc, offs) != ora_iq(v, eb_e)) bad++;
  }
  printf("%lld %lld\n", checked, bad);
  return bad ? 1 : 0;
}
