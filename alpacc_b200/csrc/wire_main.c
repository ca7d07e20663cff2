/*
 * Wire-protocol program around the B200 path (docs/wire-protocols.md of
 * alpacc): the same interface as a generated combined-, lexer- or
 * parser-mode program
 * (backends/c/cli.c) — counted batches of frames on stdin, one response
 * record per frame on stdout, `--server` loops over batches until EOF with a
 * flush after every record, `--layout` prints the native type sizes.
 *
 * This file is compiled after a grammar's constants and the glue that builds
 * `alpacc_tables` from them and defines
 *   static alpacc_gpu_grammar *gpu_grammar(void);
 * (see alpacc_b200/wire_program.py, which assembles the source).
 *
 * Frame errors (truncated input, frame_len mismatch) end the program with exit
 * status 1 as the reference's program does; an internal GPU error also exits
 * with status 1 and a message, instead of being written as a reject.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static int read_u64(FILE *f, uint64_t *v) { return fread(v, sizeof *v, 1, f) == 1; }

static void write_u64(FILE *f, uint64_t v) { fwrite(&v, sizeof v, 1, f); }

/* 0 ok, -1 frame error */
static int one_frame(FILE *in, FILE *out) {
  uint64_t frame_len;
  if (!read_u64(in, &frame_len)) {
    fprintf(stderr, "error: truncated input\n");
    return -1;
  }
  if (frame_len < 8) {
    fprintf(stderr, "error: bad frame length\n");
    return -1;
  }
  uint8_t *frame = (uint8_t *)malloc(frame_len);
  if (!frame || fread(frame, 1, frame_len, in) != frame_len) {
    fprintf(stderr, "error: truncated frame\n");
    free(frame);
    return -1;
  }
  uint64_t n;
  memcpy(&n, frame, 8);
  if (n > (frame_len - 8) / WIRE_UNIT || n * WIRE_UNIT != frame_len - 8) {
    fprintf(stderr, "error: frame length mismatch\n");
    free(frame);
    return -1;
  }
  int rc = alpacc_gpu_run_case(gpu_grammar(), n, frame + 8, out);
  free(frame);
  if (rc < 0) {
    fprintf(stderr, "error: %s\n", alpacc_strerror(rc));
    exit(1);
  }
  return 0;
}

/* 0 ok, 1 clean EOF before the count (server mode), -1 error */
static int one_batch(FILE *in, FILE *out, int allow_eof, int flush_each) {
  uint64_t count;
  if (!read_u64(in, &count)) {
    if (allow_eof && feof(in)) return 1;
    fprintf(stderr, "error: truncated input\n");
    return -1;
  }
  write_u64(out, count);
  for (uint64_t i = 0; i < count; i++) {
    if (one_frame(in, out) != 0) return -1;
    if (flush_each) fflush(out);
  }
  return 0;
}

static void usage(const char *p) {
  fprintf(stderr,
          "Usage: %s [options]\n"
          "  -i FILE    input file  (default: stdin)\n"
          "  -o FILE    output file (default: stdout)\n"
          "  --timeit   print wall-clock elapsed time to stderr\n"
          "  --server   counted-batch loop until EOF (flush per response)\n"
          "  --layout   print native type sizes and exit\n"
          "  -h/--help  show this message\n",
          p);
}

int main(int argc, char **argv) {
  const char *ifile = NULL, *ofile = NULL;
  int timeit = 0, server = 0;
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "-h") || !strcmp(argv[i], "--help")) {
      usage(argv[0]);
      return 0;
    } else if (!strcmp(argv[i], "--timeit")) {
      timeit = 1;
    } else if (!strcmp(argv[i], "--server")) {
      server = 1;
    } else if (!strcmp(argv[i], "--layout")) {
      print_layout(stdout);  /* from the types in scope: no device needed */
      return 0;
    } else if (!strcmp(argv[i], "-i") && i + 1 < argc) {
      ifile = argv[++i];
    } else if (!strcmp(argv[i], "-o") && i + 1 < argc) {
      ofile = argv[++i];
    } else {
      fprintf(stderr, "error: unknown argument '%s'\n", argv[i]);
      usage(argv[0]);
      return 1;
    }
  }
  FILE *in = stdin, *out = stdout;
  if (ifile && !(in = fopen(ifile, "rb"))) {
    perror(ifile);
    return 1;
  }
  if (ofile && !(out = fopen(ofile, "wb"))) {
    perror(ofile);
    return 1;
  }
  struct timespec t0, t1;
  if (timeit) clock_gettime(CLOCK_MONOTONIC, &t0);
  int rc;
  if (server) {
    for (;;) {
      int r = one_batch(in, out, 1, 1);
      if (r == 1) {
        rc = 0;
        break;
      }
      if (r < 0) {
        rc = 1;
        break;
      }
      fflush(out);
    }
  } else {
    rc = one_batch(in, out, 0, 0) == 0 ? 0 : 1;
    fflush(out);
  }
  if (timeit) {
    clock_gettime(CLOCK_MONOTONIC, &t1);
    fprintf(stderr, "Time: %.2fms\n", (t1.tv_sec - t0.tv_sec) * 1e3 + (t1.tv_nsec - t0.tv_nsec) * 1e-6);
  }
  if (in != stdin) fclose(in);
  if (out != stdout) fclose(out);
  return rc;
}
