/*
 * alpacc_b200 — C ABI of the B200 (sm_100a) lex + LLP-parse path.
 *
 * A drop-in for the combined-mode ``run_case`` of a program generated by
 * alpacc (CoderDue/alpacc): bytes in, and either reject or the token sequence
 * with spans plus the preorder production tree with parent indices out.
 *
 * Reference interfaces replaced (paths within the alpacc project):
 *   - the grammar constants a generated program bakes in, emitted by
 *     src/Alpacc/Generator/C/Lexer.hs:16-58 (TO_STATE, COMPOSE, ACCEPT, masks,
 *     IDENTITY, IGNORE_TOKEN) and src/Alpacc/Generator/C/Parser.hs:21-95
 *     (Q, K, sentinels, hash table, STACKS, PRODUCTIONS, arities,
 *     PRODUCTION_TO_TERMINAL_IS_VALID)                  -> alpacc_tables
 *   - the per-input device set-up of the CUDA backend
 *     (backends/cuda/cli.cu:739-792 ``both_one``, lexer.cu:274-302 ``LexerCtx``,
 *     parser.cu:700-811 ``allocParserFused``)           -> alpacc_gpu_load
 *   - ``run_case(uint64_t n, const uint8_t *in, FILE *out)``
 *     (src/Alpacc/Generator/C/Generator.hs:114-152)      -> alpacc_gpu_run_case
 *     and its in-memory form                            -> alpacc_gpu_parse
 *   - the lexer-mode and parser-mode ``run_case`` (C/Generator.hs:64-108) and
 *     the CUDA backend's ``lex_one`` / ``runParserPipeline``
 *     (backends/cuda/cli.cu:237-275, 513-526)  -> alpacc_gpu_lex,
 *                                                  alpacc_gpu_parse_tokens
 *   - ``print_layout`` (C/Generator.hs:153-158, cli.c --layout)
 *                                                       -> alpacc_gpu_layout
 *
 * Results are bit-identical to the reference's C backend (backends/c/lexer.c,
 * backends/c/parser.c) on the same tables and input. Unlike the reference,
 * errors (CUDA failure, allocation failure, a device wait that timed out, an
 * input beyond capacity) are reported as negative status codes and never as
 * a reject.
 */
#ifndef ALPACC_B200_H
#define ALPACC_B200_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALPACC_ABI_VERSION 1

/* Status codes. */
#define ALPACC_OK 0          /* input accepted, result filled */
#define ALPACC_REJECT 1      /* input rejected (the reference writes byte 0) */
#define ALPACC_E_INVALID (-1)  /* bad argument or malformed tables */
#define ALPACC_E_CUDA (-2)     /* a CUDA call failed */
#define ALPACC_E_NOMEM (-3)    /* device or pinned allocation failed */
#define ALPACC_E_CAPACITY (-4) /* input larger than the configured capacity */
#define ALPACC_E_TIMEOUT (-5)  /* a bounded device wait gave up */
#define ALPACC_E_UNSUPPORTED (-6) /* tables exceed what the kernels handle */
#define ALPACC_E_ABORTED (-7)  /* a caller's callback asked to stop */

/*
 * Which tables a generated program holds (src/Alpacc/Generator/C/Generator.hs:
 * 161-201): the combined program has both, the lexer-mode program only the
 * lexer constants (with the lexer's own terminal numbering, mkLexer in
 * src/Alpacc/Generator/Analyzer.hs:114-150), the parser-mode program only
 * the parser constants without the tree section (no arities: the
 * production_to_* pointers are NULL and number_of_productions is 0). Fields
 * of the absent part are ignored.
 */
#define ALPACC_PARTS_BOTH 0
#define ALPACC_PARTS_LEXER 1
#define ALPACC_PARTS_PARSER 2

/*
 * Grammar tables exactly as alpacc's C emitter produces them. Element widths
 * are given in bytes; arrays use those native widths, little-endian.
 */
typedef struct alpacc_tables {
  uint32_t abi_version;        /* ALPACC_ABI_VERSION */
  uint32_t terminal_size;      /* sizeof(terminal_t)   */
  uint32_t production_size;    /* sizeof(production_t) */
  uint32_t bracket_size;       /* sizeof(bracket_t)    */
  uint32_t state_size;         /* sizeof(state_t)      */
  uint32_t index_size;         /* sizeof(index_t): 4 (--index32) or 8 */
  uint32_t length_size;        /* sizeof(length_t)     */
  uint32_t parts;              /* ALPACC_PARTS_*: which program the tables come from */
  /* lexer: C/Lexer.hs:16-58 */
  uint64_t num_states;         /* NUM_STATES (endomorphisms) */
  uint64_t endo_mask, endo_offset;
  uint64_t terminal_mask, terminal_offset;
  uint64_t produce_mask, produce_offset;
  uint64_t identity;           /* IDENTITY */
  int64_t ignore_token;        /* IGNORE_TOKEN, or -1 when the grammar has none */
  const void *to_state;        /* state_t[256]                      TO_STATE */
  const void *compose;         /* state_t[num_states * num_states]  COMPOSE  */
  const uint8_t *accept;       /* bool[num_states]                  ACCEPT   */
  /* parser: C/Parser.hs:21-95 */
  uint64_t q, k;               /* Q, K */
  uint64_t empty_terminal, start_terminal, end_terminal;
  uint64_t hash_table_size;    /* HASH_TABLE_SIZE */
  uint64_t max_iters;          /* MAX_ITERS */
  uint64_t stacks_size, productions_size;
  uint64_t max_brackets_per_position, max_prods_per_position;
  const void *stacks;          /* bracket_t[stacks_size]            STACKS */
  const void *productions;     /* production_t[productions_size]    PRODUCTIONS */
  const uint8_t *hash_table_is_valid;        /* bool[hash_table_size] */
  const void *hash_table_keys;               /* terminal_t[hash_table_size][q + k] */
  const int64_t *hash_table_stacks_span;     /* int64_t[hash_table_size][2] */
  const int64_t *hash_table_productions_span;/* int64_t[hash_table_size][2] */
  uint64_t number_of_productions;            /* NUMBER_OF_PRODUCTIONS */
  const uint64_t *production_to_arity;       /* uint64_t[number_of_productions] */
  const uint8_t *production_to_terminal_is_valid; /* bool[number_of_productions] */
} alpacc_tables;

/* Opaque handle: the grammar's device tables, a stream and resident scratch. */
typedef struct alpacc_gpu_grammar alpacc_gpu_grammar;

/*
 * Result of one parse (SoA, native widths; matches the combined-mode record of
 * docs/wire-protocols.md). Host results live in library-owned pinned memory
 * released by alpacc_result_free; device results point into the grammar's
 * resident scratch and stay valid until the next call on that handle.
 */
typedef struct alpacc_result {
  uint8_t valid;               /* 1 accepted, 0 rejected */
  uint8_t on_device;           /* 1 when the arrays are device pointers */
  uint16_t reserved0;
  uint32_t reserved1;
  uint64_t num_tokens;
  uint64_t num_nodes;
  void *token_ids;             /* terminal_t[num_tokens] */
  void *token_starts;          /* index_t[num_tokens]    */
  void *token_lengths;         /* length_t[num_tokens]   */
  void *node_productions;      /* production_t[num_nodes] (preorder) */
  void *node_parents;          /* index_t[num_nodes]     */
  void *token_parents;         /* index_t[num_tokens]    */
  void *internal;              /* owned buffer, freed by alpacc_result_free */
} alpacc_result;

/*
 * Upload the tables of one grammar to `device` once and derive the device
 * forms (the minimised lexer automaton, the pair-lookup table). `max_input`
 * bytes of scratch capacity are reserved up front (0 = grow on demand).
 * Returns NULL and sets *err on failure.
 */
alpacc_gpu_grammar *alpacc_gpu_load(const alpacc_tables *tables, int device, uint64_t max_input, int *err);

/* Release the handle, its device tables and its scratch. */
void alpacc_gpu_free(alpacc_gpu_grammar *g);

/*
 * Parse host bytes: H2D copy, the device path, D2H copy of the result into
 * pinned memory owned by *out. The input is copied in pieces of ~16 MiB and
 * each piece is lexed as soon as it has arrived; the token arrays are copied
 * back while the parser runs. Returns ALPACC_OK, ALPACC_REJECT or an error.
 */
int alpacc_gpu_parse(alpacc_gpu_grammar *g, const uint8_t *in, uint64_t n, alpacc_result *out);

/*
 * Parse bytes already resident on the device (`d_in`, n bytes) on the
 * handle's stream; the result arrays are device pointers into the handle's
 * scratch (out->on_device = 1). Blocks until the status is known.
 */
int alpacc_gpu_parse_device(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, alpacc_result *out);

/*
 * Lex device-resident bytes into caller-provided device arrays (terminal_t,
 * index_t and length_t, room for n tokens each) without allocating anything
 * at call time. This entry point has no counterpart in the reference. It is
 * for callers that must not call cudaMalloc where they lex: a host framework
 * whose caching allocator owns the device memory, or a real-time loop that
 * cannot take the allocator's locks or wait on its synchronisation. The
 * lexer's working memory is a fixed array inside the library, sized for
 * inputs of at most 16 MiB (larger n returns ALPACC_E_CAPACITY). Every call
 * shares that array, so calls must not overlap on the GPU (two streams, two
 * threads or two handles on one device race on it); the array's address is
 * looked up on the first call on each device, which should therefore come
 * before any stream capture. Every call, the first and the later ones, ends
 * by copying the status words back and waiting for the handle's stream
 * (cudaStreamSynchronize) before it returns. The call makes the handle's
 * device current while it runs and restores the caller's current device
 * before returning. Returns ALPACC_OK with *num_tokens set, ALPACC_REJECT, or
 * an error.
 */
int alpacc_gpu_lex_noalloc(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, void *d_token_ids,
                           void *d_token_starts, void *d_token_lengths, uint64_t *num_tokens);

/*
 * Run the device path for device-resident input (as alpacc_gpu_parse_device,
 * which also waits for the status) and keep the outcome in the handle;
 * alpacc_gpu_collect then returns that status and the device result arrays.
 */
int alpacc_gpu_enqueue(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n);
int alpacc_gpu_collect(alpacc_gpu_grammar *g, alpacc_result *out);

/*
 * Many independent inputs at once: `bytes` holds them back to back, input i is
 * bytes[offsets[i] .. offsets[i+1]). `outs` receives `count` results, each
 * identical to parsing that input alone. Every stage is launched once for the
 * whole batch (the reference sets up and launches per input,
 * backends/cuda/cli.cu:739-792); the results share one pinned block, released
 * when the last of them is passed to alpacc_result_free. Returns ALPACC_OK
 * when every input was processed (each outs[i].valid says accept/reject) or
 * the first error.
 */
int alpacc_gpu_parse_batch(alpacc_gpu_grammar *g, const uint8_t *bytes, const int64_t *offsets, uint32_t count,
                           alpacc_result *outs);

/* Release a host result. Its pinned block returns to the handle for reuse, so
   results must be released before the handle that produced them. */
void alpacc_result_free(alpacc_result *r);

/*
 * Request server with continuous batching (replaces the reference's
 * sequential `--server` loop, backends/c/cli.c:153-161 and
 * backends/cuda/cli.cu:846-875, for in-process callers). `workers` threads each
 * own a handle and a stream; a free worker takes queued requests, in order,
 * while the exact device scratch of their batch (the sizes the batch path
 * grows its buffers to) stays within its share (scratch_budget / workers), and
 * parses them as one batch, so requests arriving while a batch runs join the
 * next one and batches overlap on the device. A worker's handle never holds
 * more batch scratch than its share, except while a single request that needs
 * more on its own runs. Each result equals parsing its input alone.
 *   submit: copies the input, returns its id;
 *   wait:   blocks until that request is done; its status (OK / REJECT /
 *           error), its result (release with alpacc_result_free before
 *           stopping the server) and the latency from submit to completion.
 *           One caller may wait for an id; a second wait on the same id
 *           (concurrent or later) returns ALPACC_E_INVALID;
 *   stats:  batches run, requests served, largest batch, requests queued,
 *           most batch scratch bytes a worker's handle held, the per-worker
 *           share (returns the number of values, 6; fills at most n);
 *   stop:   drains the queue, joins the workers, frees the handles.
 */
typedef struct alpacc_server alpacc_server;
alpacc_server *alpacc_server_start(const alpacc_tables *tables, int device, int workers, uint64_t scratch_budget,
                                   int *err);
int alpacc_server_submit(alpacc_server *s, const uint8_t *in, uint64_t n, uint64_t *id);
int alpacc_server_wait(alpacc_server *s, uint64_t id, alpacc_result *out, double *latency_ms);
int alpacc_server_stats(alpacc_server *s, int64_t *vals, int n);
void alpacc_server_stop(alpacc_server *s);

/*
 * Trace replay, for measuring the served form against plain calls (no
 * counterpart in the reference). Request i is input doc[i] of a pool
 * (bytes[offsets[k]..offsets[k+1]) is input k) arriving arrival_s[i] seconds
 * after the call starts (non-decreasing). alpacc_server_replay submits each
 * at its arrival from a native thread and waits for all in order;
 * alpacc_gpu_replay makes one alpacc_gpu_parse per request on g, in order,
 * none before its arrival. Both release every result and fill, per request,
 * status[i] (OK, REJECT or an error) and latency_ms[i] (scheduled arrival to
 * result), and *elapsed_s (start to the last result).
 */
int alpacc_server_replay(alpacc_server *s, const uint8_t *bytes, const int64_t *offsets, const uint32_t *doc,
                         uint64_t count, const double *arrival_s, double *latency_ms, int *status,
                         double *elapsed_s);
int alpacc_gpu_replay(alpacc_gpu_grammar *g, const uint8_t *bytes, const int64_t *offsets, const uint32_t *doc,
                      uint64_t count, const double *arrival_s, double *latency_ms, int *status, double *elapsed_s);

/*
 * Lexer-only mode: the lexemes of lex_string (backends/c/lexer.c:39-97) for
 * host bytes, as the lexer-mode program's run_case (C/Generator.hs:87-102) and
 * the CUDA backend's lex_one (backends/cuda/cli.cu:237-275) compute them.
 * Fills valid, num_tokens, token_ids, token_starts and token_lengths; the tree
 * fields stay 0 / NULL. Works on lexer-only and combined tables (token ids
 * follow the tables' own numbering).
 */
int alpacc_gpu_lex(alpacc_gpu_grammar *g, const uint8_t *in, uint64_t n, alpacc_result *out);

/*
 * Chunked lexing for inputs larger than device memory or than one device pass
 * (2^31 - 1 bytes): the counterpart of the reference's streaming chunk carry
 * (LexerCtx::update, backends/cuda/lexer.cu:224-432; lex_step, lexer.fut:96-196).
 * The host input is lexed in windows of `window` bytes (0: 1 GiB). A window
 * that ends inside the input leaves its last token open: the next window
 * starts at that token's first byte, where lex_string's state is the initial
 * one again, so the lexemes are exactly lex_string's (backends/c/lexer.c:
 * 39-97). A window in which no token ends is doubled and lexed again (up to
 * 2^31 - 1 bytes, else ALPACC_E_CAPACITY). After each window `sink` receives
 * its lexemes (host arrays of `count` terminal_t ids, index_t absolute
 * starts and length_t lengths, valid during the call; `first` = index of the
 * first one); a nonzero return stops with ALPACC_E_ABORTED. Returns
 * ALPACC_OK with *num_tokens set, ALPACC_REJECT (lexemes already passed to
 * the sink are then void), or an error. Tables with 32-bit index_t take at
 * most 2^31 - 1 bytes.
 */
typedef int (*alpacc_lex_sink)(void *user, uint64_t first, uint64_t count, const void *token_ids,
                               const void *token_starts, const void *token_lengths);
int alpacc_gpu_lex_stream(alpacc_gpu_grammar *g, const uint8_t *in, uint64_t n, uint64_t window,
                          alpacc_lex_sink sink, void *user, uint64_t *num_tokens);

/*
 * Parser-only mode: `tokens` holds n terminal_t ids (host memory); the result
 * is parse_test's production sequence (backends/c/parser.c:49-98; the
 * parser-mode run_case, C/Generator.hs:65-79; runParserPipeline of
 * backends/cuda/cli.cu:513-526): valid, num_nodes = number of productions,
 * node_productions = production_t[num_nodes] in derivation order (not
 * compacted); the token and parent fields stay 0 / NULL. Works on parser-only
 * and combined tables.
 */
int alpacc_gpu_parse_tokens(alpacc_gpu_grammar *g, const void *tokens, uint64_t n, alpacc_result *out);

/*
 * Write the response record of the handle's mode for one input to `out`, byte
 * for byte what the generated run_case writes (u8 valid, then when valid):
 *   combined tables: the token and tree sections (C/Generator.hs:114-152),
 *     `in` = n bytes;
 *   lexer-only tables: u64 count, then per lexeme terminal_t, index_t start,
 *     length_t length (C/Generator.hs:87-102), `in` = n bytes;
 *   parser-only tables: u64 count, then production_t ids
 *     (C/Generator.hs:65-79), `in` = n terminal_t ids.
 * Returns the status of the call.
 */
int alpacc_gpu_run_case(alpacc_gpu_grammar *g, uint64_t n, const uint8_t *in, FILE *out);

/* `--layout` text of the handle's mode ("terminal_t=1\nproduction_t=1\n...",
   the lines print_layout writes in that mode); returns its length. */
int alpacc_gpu_layout(const alpacc_gpu_grammar *g, char *buf, size_t len);

/* Human-readable text of a status code. */
const char *alpacc_strerror(int status);

/*
 * Device time of the last enqueued device path in milliseconds (CUDA events
 * around the launches on the handle's stream), or a negative value.
 */
double alpacc_gpu_last_ms(alpacc_gpu_grammar *g);

/*
 * Autotuner (no counterpart in the reference, whose CUDA backend takes its
 * launch shapes from per-architecture tables, backends/cuda/lexer.cu:101-193,
 * backends/cuda/parser.cu:82-136): times the device-resident sample under each
 * candidate launch geometry and keeps the fastest for this handle's grammar -
 * first the lexer's window before each chunk (16, 24 or 32 bytes) with its
 * resident CTAs per SM (the occupancy limit and up to two below it), then
 * (combined tables) the pair kernel's and then the depth walks' resident
 * CTAs per SM, each on its own stages' device time. The choice is cached for
 * the process per (grammar, device): handles loaded afterwards for the same
 * tables on the same device start with it. *choice receives the lexer's CTAs
 * per SM. The call synchronises with the handle's stream.
 */
int alpacc_gpu_autotune(alpacc_gpu_grammar *g, const uint8_t *d_sample, uint64_t n, int *choice);

/* The handle's launch geometry: lexer window bytes, lexer / pair / walk
   resident CTAs per SM, whether it came from the autotuner's cache at load,
   the grammar digest that keys that cache. Returns the number of values (6). */
int alpacc_gpu_geometry(const alpacc_gpu_grammar *g, int64_t *vals, int n);

/* The cudaStream_t the handle launches on, so a caller can order its own work
   (copies, events) with it. */
void *alpacc_gpu_stream(alpacc_gpu_grammar *g);

/*
 * Diagnostics (no counterpart in the reference): sizes of the derived device
 * tables (states and byte classes of the minimised lexer automaton, lanes,
 * reachable endomorphisms, pair records), the lexer's grid, the reject reason /
 * wait site of the last call, whether the pair table is in its hashed form,
 * the lexer kernel variant (0 / 1: window machine for machines of at most /
 * more than 64 states, 2: windows walked as explicit state sets) and the
 * window machine's sets (0: not built); and the text of the last internal
 * error.
 *
 * The pair table is a dense array for key spaces up to 2^26 keys and the
 * reference's own hash table, probed on the device as lookup_key probes it,
 * beyond; ALPACC_PAIR_LOOKUP=hashed in the environment at load time selects
 * the hashed form for any grammar (for checking it). Likewise
 * ALPACC_LEX_WINDOW=sets selects the explicit state-set window walk.
 */
int alpacc_gpu_info(const alpacc_gpu_grammar *g, int64_t *vals, int nvals);
const char *alpacc_gpu_last_error(const alpacc_gpu_grammar *g);
/* Device time of each stage of the last call (ms): lexer, pair expansion,
   bracket walk, bracket resolve, parent walk, parent resolve; zeros unless
   stage timing is on (alpacc_gpu_set_stage_timing, off by default: its event
   records cost a small input's call host time). */
int alpacc_gpu_stage_ms(const alpacc_gpu_grammar *g, double *out, int n);
void alpacc_gpu_set_stage_timing(alpacc_gpu_grammar *g, int on);
/* Tokens, brackets, productions and tree nodes of the last call, then four
   lexer diagnostic counters (collected when diagnostics are on): tiles that
   read their incoming state from the previous tile, chunks whose start state
   their window settled, chunk evaluations chained to find the other chunks'
   start states, candidate walks of those chunks; then the number of kernels
   the call launched; then (diagnostics on) the SM cycles thread 0 of the
   lexer's CTAs spent in each phase, summed over tiles: load, window walk,
   chunk and candidate walks, known-chunk scan, start states, open chunks'
   codes with the masks and the count scan, the count look-back, the token or
   code writes; then the same for the bracket walk's and the parent walk's
   tile kernel: load with steps and scan, depths and windows, own and previous
   chunk queries, the warps' queued queries, look-back, staircase and
   unanswered queries, tree entries, next tile. Returns the number of values
   (33). */
int alpacc_gpu_counts(const alpacc_gpu_grammar *g, int64_t *vals, int n);
void alpacc_gpu_set_diagnostics(alpacc_gpu_grammar *g, int on);
/* Number of device allocations (cudaMalloc) this library has made in the
   process so far, over all handles (diagnostics: lets a caller check that a
   call allocated nothing). */
uint64_t alpacc_device_allocations(void);

#ifdef __cplusplus
}
#endif

#endif /* ALPACC_B200_H */
