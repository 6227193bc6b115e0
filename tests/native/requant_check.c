/* Exhaustive check of the shift form of requantization used by the
 * re-encoders' fast path (init_send, resi_send) against the oracle's
 * composition of the reference quantizers (iSQ -> CQ; and CQ -> iCQ -> CQ for
 * residuals).  Test infrastructure only: links the CPU oracle.
 *
 * Build: gcc -O2 -fopenmp requant_check.c -L<oracle> -lcortado_oracle
 * Usage: requant_check <mode 0=init 1=resi> <e_s> <e_1> <e_2> <full 0/1>
 * Prints the number of checked words and mismatches; exit status 1 on any
 * mismatch. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

uint32_t ora_cq(uint32_t v, int eb_e);
uint32_t ora_iq(uint32_t v, int eb_e);

/* PTX shl.b32 / shr.b32: shift amounts of 32 or more (as unsigned) give 0. */
static uint32_t shl_c(uint32_t x, uint32_t s) { return s >= 32 ? 0u : x << s; }
static uint32_t shr_c(uint32_t x, uint32_t s) { return s >= 32 ? 0u : x >> s; }
/* round-half-away-from-zero division of a magnitude by 2^k (k >= 0) */
static uint32_t rq(uint32_t a, int k) { return shr_c(a + shl_c(1u, (uint32_t)(k - 1)), (uint32_t)k); }

/* returns 1 and the result when the fast path applies to stored bin v; the
 * decision is the device's: every magnitude below a bound that depends only
 * on the exponents.  *disagree is set when the direct test of the shifted
 * source bin (m1 << d must stay a lossy destination bin) decides otherwise. */
static int fast(int mode, uint32_t v, int es, int e1, int e2, uint32_t* out, int* disagree) {
  const int k1 = e1 - es, k2 = mode ? e2 - es : 0, d = mode ? e1 - e2 : 0;
  const uint32_t neg = (uint32_t)((int32_t)v >> 31);
  const uint32_t a = (v ^ neg) - neg;
  if (k1 < 0 || k2 < 0 || d < 0) return 0;
  const uint32_t amax = (mode && k2 == 0 && k1 >= 1 && k1 <= 23) ? 0x800000u - (1u << (k1 - 1)) : 0x800000u;
  const int ok = a < amax;
  if (mode && a < 0x800000u) {
    const uint32_t m1 = rq(a, k1);
    const int direct = d > 23 ? m1 == 0 : m1 < (0x800000u >> d);
    if (direct != ok) *disagree = 1;
  }
  if (!ok) return 0;
  const uint32_t m1 = rq(a, k1);
  const uint32_t r = mode ? rq(a, k2) - shl_c(m1, (uint32_t)d) : m1;
  *out = (r ^ neg) - neg;
  return 1;
}

static uint32_t slow(int mode, uint32_t v, int es, int e1, int e2) {
  const uint32_t x = ora_iq(v, es);
  if (mode == 0) return ora_cq(x, e1);
  const uint32_t src_req = ora_cq(ora_iq(ora_cq(x, e1), e1), e2);
  return ora_cq(x, e2) - src_req;
}

int main(int argc, char** argv) {
  if (argc < 6) return 2;
  const int mode = atoi(argv[1]), es = atoi(argv[2]), e1 = atoi(argv[3]), e2 = atoi(argv[4]), full = atoi(argv[5]);
  long long checked = 0, bad = 0, fastn = 0;
  const uint32_t top = full ? 0x800000u : 0x10000u;
#pragma omp parallel for reduction(+ : checked, bad, fastn) schedule(static)
  for (long long i = 0; i < (long long)top; i++) {
    uint32_t as[6];
    int n = 0;
    as[n++] = (uint32_t)i;
    if (!full) {
      /* beyond 2^16: every value within 3 of a power of two, and a spread */
      const uint32_t p = 1u << (16 + (i & 7)), r = (uint32_t)(i >> 3);
      as[n++] = (p + (r & 7) - 3) & 0x7fffffu;
      as[n++] = (uint32_t)((i * 2654435761ull) & 0x7fffffu);
      as[n++] = 0x7fffffu - (uint32_t)(i & 0xff);
    }
    as[n++] = 0x800000u + (uint32_t)(i & 0xfff); /* lossless bins: must leave the fast path */
    for (int j = 0; j < n; j++) {
      for (int sgn = 0; sgn < 2; sgn++) {
        const uint32_t v = sgn ? (uint32_t)(-(int32_t)as[j]) : as[j];
        uint32_t f;
        int disagree = 0;
        checked++;
        if (fast(mode, v, es, e1, e2, &f, &disagree)) {
          fastn++;
          if (f != slow(mode, v, es, e1, e2)) bad++;
        }
        if (disagree) bad++;
      }
    }
  }
  printf("%lld %lld %lld\n", checked, fastn, bad);
  return bad ? 1 : 0;
}
