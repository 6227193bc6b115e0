/*
 * Command-line drivers with the reference's arguments, files and report lines
 * (src/cortado_store.cu, src/cortado_init.cu, src/cortado_resi.cu; user mode).
 * One source, five programs selected at compile time:
 *   -DCLI_STORE      store <input> <eb...> [-o dir] [-a] [-p] [-r runs]
 *   -DCLI_INIT_SEND  init_send <server_dir> <request_eb> [-c file] [-a] [-p] [-r runs]
 *   -DCLI_INIT_RECV  init_recv <init_file> [-d file] [-p] [-r runs]
 *   -DCLI_RESI_SEND  resi_send <server_dir> <src_eb> <dst_eb> [-c file] [-a] [-p] [-r runs]
 *   -DCLI_RESI_RECV  resi_recv <src_file> <resi_file> [-d file] [-p] [-r runs]
 * Error bounds are NOA (normalized by max-min) unless -a is given.
 * Host-only logic: argument parsing, bound scaling (float arithmetic, as the
 * reference compiles with -ffp-contract=off), .stor.meta, stored-file choice.
 */
#define _XOPEN_SOURCE 700 /* nftw */
#include <cuda_runtime.h>
#include <errno.h>
#include <ftw.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "../../include/cortado.h"

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { fprintf(stderr, "CUDA error %d on line %d: %s\n\n", (int)e_, __LINE__, cudaGetErrorString(e_)); exit(1); } } while (0)
#define CS_(x, what) do { cortado_status s_ = (x); if (s_ != CORTADO_OK) { fprintf(stderr, "ERROR: %s: %s\n", what, cortado_status_string(s_)); exit(1); } } while (0)

static int remove_entry(const char* path, const struct stat* sb, int flag, struct FTW* ftw) {
  (void)sb;
  (void)flag;
  (void)ftw;
  return remove(path); /* files, links, and directories once emptied (depth first) */
}

/* Deletes `dir` with everything in it, then creates it again with any missing
 * parents: the reference's std::filesystem::remove_all + create_directories
 * (src/cortado_store.cu:170-179), without a shell, so no character of the path
 * is interpreted. */
static int reset_dir(const char* dir) {
  struct stat st;
  if (lstat(dir, &st) == 0 && nftw(dir, remove_entry, 64, FTW_DEPTH | FTW_PHYS) != 0) return -1;
  char buf[4096];
  const size_t n = strlen(dir);
  if (n == 0 || n >= sizeof buf) return -1;
  memcpy(buf, dir, n + 1);
  for (char* p = buf + 1; *p; p++) {
    if (*p != '/') continue;
    *p = 0;
    if (mkdir(buf, 0777) != 0 && errno != EEXIST) return -1;
    *p = '/';
  }
  if (mkdir(buf, 0777) != 0 && errno != EEXIST) return -1;
  return 0;
}

static unsigned char* read_file(const char* name, long long* size) {
  FILE* f = fopen(name, "rb");
  if (!f) { fprintf(stderr, "ERROR: cannot open %s\n\n", name); exit(1); }
  fseek(f, 0, SEEK_END);
  long long n = ftell(f);
  if (n <= 0) { fprintf(stderr, "ERROR: input file too small\n\n"); exit(1); }
  unsigned char* b = (unsigned char*)malloc((size_t)n);
  fseek(f, 0, SEEK_SET);
  if ((long long)fread(b, 1, (size_t)n, f) != n) { fprintf(stderr, "ERROR: short read on %s\n", name); exit(1); }
  fclose(f);
  *size = n;
  return b;
}

static void write_file(const char* name, const void* data, long long n) {
  FILE* f = fopen(name, "wb");
  if (!f || (long long)fwrite(data, 1, (size_t)n, f) != n) { fprintf(stderr, "ERROR: cannot write %s\n", name); exit(1); }
  fclose(f);
}

static const char* base_name(const char* p) {
  const char* s = strrchr(p, '/');
  return s ? s + 1 : p;
}

static int cmp_desc(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x < y) - (x > y);
}

static double median(double* v, int n) {
  for (int i = 1; i < n; i++)
    for (int j = i; j > 0 && v[j - 1] > v[j]; j--) { double t = v[j]; v[j] = v[j - 1]; v[j - 1] = t; }
  return (n % 2 == 0) ? (v[(n - 1) / 2] + v[n / 2]) / 2.0 : v[n / 2];
}

/* util.h:101-135 */
static void read_meta(const char* dir, char** name, float** ebs, int* n, float* range) {
  char path[4096];
  snprintf(path, sizeof path, "%s/.stor.meta", dir);
  long long sz;
  unsigned char* b = read_file(path, &sz);
  int name_len, cnt;
  memcpy(&name_len, b, 4);
  memcpy(&cnt, b + 4, 4);
  *ebs = (float*)malloc(sizeof(float) * (size_t)(cnt > 0 ? cnt : 1));
  memcpy(*ebs, b + 8, 4 * (size_t)cnt);
  memcpy(range, b + 8 + 4 * cnt, 4);
  *name = (char*)calloc((size_t)name_len + 1, 1);
  memcpy(*name, b + 12 + 4 * cnt, (size_t)name_len);
  *n = cnt;
  free(b);
}

typedef struct {
  const char* pos[8];
  int npos;
  const char* c_out;
  const char* d_out;
  const char* o_dir;
  int abs_mode, perf, runs;
} args_t;

static void usage(const char* prog) {
  fprintf(stderr, "usage: %s <positional args> [-o dir] [-c file] [-d file] [-a] [-p] [-r runs] [-h]\n", prog);
}

static args_t parse(int argc, char** argv) {
  args_t a;
  memset(&a, 0, sizeof a);
  a.runs = 1;
  for (int i = 1; i < argc; i++) {
    const char* s = argv[i];
    if (!strcmp(s, "-h") || !strcmp(s, "--help")) { usage(argv[0]); exit(0); }
    else if (!strcmp(s, "-a") || !strcmp(s, "--abs")) a.abs_mode = 1;
    else if (!strcmp(s, "-p") || !strcmp(s, "--perf")) a.perf = 1;
    else if ((!strcmp(s, "-r") || !strcmp(s, "--runs")) && i + 1 < argc) a.runs = atoi(argv[++i]);
    else if ((!strcmp(s, "-o") || !strcmp(s, "--output_dir")) && i + 1 < argc) a.o_dir = argv[++i];
    else if ((!strcmp(s, "-c") || !strcmp(s, "--compressed_output")) && i + 1 < argc) a.c_out = argv[++i];
    else if ((!strcmp(s, "-d") || !strcmp(s, "--decompressed_output")) && i + 1 < argc) a.d_out = argv[++i];
    else if (a.npos < 8) a.pos[a.npos++] = s;
  }
  if (a.runs > 1) a.perf = 1;
  if (!a.perf) a.runs = 1;
  return a;
}

static float parse_eb(const char* s) { return strtof(s, NULL); }

static void report(const char* what, long long insize, double runtime, int perf) {
  if (perf) {
    printf("%s runtime:    %.6f s\n", what, runtime);
    printf("%s throughput: %.3f Gbytes/s\n", what, insize * 0.000000001 / runtime);
  }
}


int main(int argc, char** argv) {
  args_t a = parse(argc, argv);
  cortado_ctx* ctx;
  CS_(cortado_create(&ctx, 0), "context");
  struct cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, 0));
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  long long* d_size;
  CK(cudaMalloc((void**)&d_size, sizeof(long long)));
  double* times = (double*)malloc(sizeof(double) * (size_t)(a.runs > 0 ? a.runs : 1));
  printf("[info]\nGPU: %s\n", prop.name);

#if defined(CLI_STORE)
  if (a.npos < 2) { usage(argv[0]); return 1; }
  const char* input = a.pos[0];
  int neb = a.npos - 1;
  float* ebs = (float*)malloc(sizeof(float) * (size_t)neb);
  for (int i = 0; i < neb; i++) ebs[i] = parse_eb(a.pos[1 + i]);
  qsort(ebs, (size_t)neb, sizeof(float), cmp_desc);
  int k = 0;
  for (int i = 0; i < neb; i++) if (i == 0 || ebs[i] != ebs[k - 1]) ebs[k++] = ebs[i];
  neb = k;
  printf("%s error bounds (%d):\n", a.abs_mode ? "ABS" : "NOA", neb);
  for (int i = 0; i < neb; i++) printf("  %lf\n", ebs[i]);
  if (a.o_dir && reset_dir(a.o_dir) != 0) {
    fprintf(stderr, "FILESYSTEM ERROR: %s\n", a.o_dir);
    return 1;
  }
  long long insize;
  unsigned char* h_in = read_file(input, &insize);
  printf("original size: %lld bytes\n", insize);
  const long long maxsize = cortado_max_stream_bytes(insize);
  void *d_in, *d_out;
  CK(cudaMalloc(&d_in, (size_t)insize));
  CK(cudaMemcpy(d_in, h_in, (size_t)insize, cudaMemcpyHostToDevice));
  float minf, maxf;
  CS_(cortado_noa_range(ctx, d_in, insize, &minf, &maxf, 0), "NOA range");
  printf("NOA min: %lf\nNOA max: %lf\n", minf, maxf);
  CK(cudaMalloc(&d_out, (size_t)maxsize));
  unsigned char* h_out = (unsigned char*)malloc((size_t)maxsize);
  for (int i = 0; i < neb; i++) {
    const float orig_eb = ebs[i];
    if (!a.abs_mode) ebs[i] = (maxf - minf) * orig_eb;
    const float eb = ebs[i];
    printf("\n[store eb %d/%d] orig: %lf, client: %lf, server: %lf\n", i + 1, neb, orig_eb, eb, eb / 2);
    if (a.perf) { CS_(cortado_store_encode(ctx, d_in, insize, eb, d_out, maxsize, (int64_t*)d_size, 0), "store"); CS_(cortado_sync(ctx, 0), "store"); }
    for (int r = 0; r < a.runs; r++) {
      CK(cudaEventRecord(t0, 0));
      CS_(cortado_store_encode(ctx, d_in, insize, eb, d_out, maxsize, (int64_t*)d_size, 0), "store");
      CK(cudaEventRecord(t1, 0));
      CS_(cortado_sync(ctx, 0), "store");
      float ms;
      CK(cudaEventElapsedTime(&ms, t0, t1));
      times[r] = ms * 1e-3;
    }
    long long encsize;
    CK(cudaMemcpy(&encsize, d_size, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_out, d_out, (size_t)encsize, cudaMemcpyDeviceToHost));
    printf("encoded size: %lld bytes\n", encsize);
    const float CR = (float)((100.0 * encsize) / insize);
    printf("comp ratio:   %.2f%%  %.3fx\n", CR, 100.0 / CR);
    report("", insize, median(times, a.runs), a.perf);
    if (a.o_dir) {
      char path[4200];
      snprintf(path, sizeof path, "%s/%s.stor.%02d", a.o_dir, base_name(input), i);
      write_file(path, h_out, encsize);
      printf("wrote compressed server file to %s\n", path);
    }
  }
  if (a.o_dir) {
    const int name_len = (int)strlen(input);
    const long long mlen = 8 + 4LL * neb + 4 + name_len;
    unsigned char* m = (unsigned char*)malloc((size_t)mlen);
    memcpy(m, &name_len, 4);
    memcpy(m + 4, &neb, 4);
    memcpy(m + 8, ebs, 4 * (size_t)neb);
    const float range = maxf - minf;
    memcpy(m + 8 + 4 * neb, &range, 4);
    memcpy(m + 12 + 4 * neb, input, (size_t)name_len);
    char path[4200];
    snprintf(path, sizeof path, "%s/.stor.meta", a.o_dir);
    write_file(path, m, mlen);
    printf("wrote server metadata file to %s\n", path);
  }
#elif defined(CLI_INIT_SEND) || defined(CLI_RESI_SEND)
#if defined(CLI_INIT_SEND)
  if (a.npos < 2) { usage(argv[0]); return 1; }
  float e1 = parse_eb(a.pos[1]), e2 = 0.0f;
#else
  if (a.npos < 3) { usage(argv[0]); return 1; }
  float e1 = parse_eb(a.pos[1]), e2 = parse_eb(a.pos[2]);
  if (e1 < e2) { fprintf(stderr, "ERROR: src eb must be greater than or equal to dest eb\n\n"); return 1; }
#endif
  printf("%s error bound mode\n", a.abs_mode ? "ABS" : "NOA");
  char* name;
  float* sebs;
  int n;
  float range;
  read_meta(a.pos[0], &name, &sebs, &n, &range);
  printf("server error bounds (%d):\n", n);
  for (int i = 0; i < n; i++) printf("  %lf\n", a.abs_mode ? sebs[i] : (sebs[i] / range));
  if (!a.abs_mode) { e1 *= range; e2 *= range; }
#if defined(CLI_INIT_SEND)
  const float sel = e1;
#else
  const float sel = e2;
#endif
  int idx = -1;
  for (int i = 0; i < n; i++) if (sel >= sebs[i]) { idx = i; break; }
  if (idx < 0) { fprintf(stderr, "ERROR: request eb (%lf) is too tight to be fulfilled by server (tightest eb: %lf)\n", sel, sebs[n - 1]); return 255; }
  printf("requantizing from server eb: %lf\n", a.abs_mode ? sebs[idx] : (sebs[idx] / range));
  char path[4200];
  snprintf(path, sizeof path, "%s/%s.stor.%02d", a.pos[0], base_name(name), idx);
  long long encsize;
  unsigned char* h_enc = read_file(path, &encsize);
  long long insize;
  memcpy(&insize, h_enc, 8);
  printf("original size:    %lld bytes\nserver file size: %lld bytes\n", insize, encsize);
  const long long maxsize = cortado_max_stream_bytes(insize);
  void *d_enc, *d_out;
  CK(cudaMalloc(&d_enc, (size_t)encsize));
  CK(cudaMemcpy(d_enc, h_enc, (size_t)encsize, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&d_out, (size_t)maxsize));
#if defined(CLI_INIT_SEND)
  printf("\n[init send]\n");
#define CALL() cortado_init_send(ctx, d_enc, encsize, insize, e1, d_out, maxsize, (int64_t*)d_size, 0)
#else
  printf("\n[resi send]\n");
#define CALL() cortado_resi_send(ctx, d_enc, encsize, insize, e1, e2, d_out, maxsize, (int64_t*)d_size, 0)
#endif
  if (a.perf) { CS_(CALL(), "send"); CS_(cortado_sync(ctx, 0), "send"); }
  for (int r = 0; r < a.runs; r++) {
    CK(cudaEventRecord(t0, 0));
    CS_(CALL(), "send");
    CK(cudaEventRecord(t1, 0));
    CS_(cortado_sync(ctx, 0), "send");
    float ms;
    CK(cudaEventElapsedTime(&ms, t0, t1));
    times[r] = ms * 1e-3;
  }
  long long outsize;
  CK(cudaMemcpy(&outsize, d_size, 8, cudaMemcpyDeviceToHost));
  unsigned char* h_out = (unsigned char*)malloc((size_t)outsize);
  CK(cudaMemcpy(h_out, d_out, (size_t)outsize, cudaMemcpyDeviceToHost));
  printf("encoded size:    %lld bytes\n", outsize);
  const float CR = (float)((100.0 * outsize) / insize);
  printf("comp ratio:      %.2f%% %.3fx\n", CR, 100.0 / CR);
  report("send", insize, median(times, a.runs), a.perf);
  if (a.c_out) {
    write_file(a.c_out, h_out, outsize);
    printf("wrote compressed %s file to %s\n",
#if defined(CLI_INIT_SEND)
           "initial",
#else
           "residual",
#endif
           a.c_out);
  }
#elif defined(CLI_INIT_RECV) || defined(CLI_RESI_RECV)
#if defined(CLI_INIT_RECV)
  if (a.npos < 1) { usage(argv[0]); return 1; }
  long long reqsize;
  unsigned char* h_req = read_file(a.pos[0], &reqsize);
  long long insize;
  memcpy(&insize, h_req, 8);
  printf("original size:        %lld bytes\ncompressed init size: %lld bytes\n", insize, reqsize);
  void *d_req, *d_out;
  CK(cudaMalloc(&d_req, (size_t)reqsize));
  CK(cudaMemcpy(d_req, h_req, (size_t)reqsize, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&d_out, (size_t)(insize > 0 ? insize : 4)));
  printf("\n[init recv]\n");
#define RCALL() cortado_init_recv(ctx, d_req, reqsize, d_out, insize, (int64_t*)d_size, 0)
#else
  if (a.npos < 2) { usage(argv[0]); return 1; }
  long long insize, resisize;
  unsigned char* h_src = read_file(a.pos[0], &insize);
  unsigned char* h_resi = read_file(a.pos[1], &resisize);
  printf("decompressed src size:  %lld bytes\ncompressed resi size:   %lld bytes\n", insize, resisize);
  void *d_src, *d_resi, *d_out;
  CK(cudaMalloc(&d_src, (size_t)insize));
  CK(cudaMemcpy(d_src, h_src, (size_t)insize, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&d_resi, (size_t)resisize));
  CK(cudaMemcpy(d_resi, h_resi, (size_t)resisize, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&d_out, (size_t)insize));
  printf("\n[resi recv]\n");
#define RCALL() cortado_resi_recv(ctx, d_src, insize, d_resi, resisize, d_out, insize, (int64_t*)d_size, 0)
#endif
  if (a.perf) { CS_(RCALL(), "recv"); CS_(cortado_sync(ctx, 0), "recv"); }
  for (int r = 0; r < a.runs; r++) {
    CK(cudaEventRecord(t0, 0));
    CS_(RCALL(), "recv");
    CK(cudaEventRecord(t1, 0));
    CS_(cortado_sync(ctx, 0), "recv");
    float ms;
    CK(cudaEventElapsedTime(&ms, t0, t1));
    times[r] = ms * 1e-3;
  }
  long long decsize;
  CK(cudaMemcpy(&decsize, d_size, 8, cudaMemcpyDeviceToHost));
  unsigned char* h_dec = (unsigned char*)malloc((size_t)(decsize > 0 ? decsize : 1));
  CK(cudaMemcpy(h_dec, d_out, (size_t)decsize, cudaMemcpyDeviceToHost));
  printf("decoded size:    %lld bytes\n", decsize);
  report("recv", insize, median(times, a.runs), a.perf);
  if (a.d_out) {
    write_file(a.d_out, h_dec, decsize);
    printf("wrote decompressed file to %s\n", a.d_out);
  }
#endif
  cortado_destroy(ctx);
  return 0;
}
