// Lexing with no allocation at call time, for callers that must not allocate.
//
// Some callers cannot call cudaMalloc on the path where they lex: code that
// runs while device memory is reserved up front by a host framework (its own
// caching allocator owns the pool and a stray cudaMalloc would fragment or
// oversubscribe it), or a real-time loop that must not take the allocator's
// locks or block on its synchronisation. For them this entry point lexes a
// device-resident input into caller-provided token arrays, with the lexer's
// working memory (tile tickets, look-back flags and carries, the status
// words) in a fixed array compiled into this library instead of allocated.
//
// Limits and sharing:
//  * the array holds the working memory for inputs of at most
//    kNoAllocMaxInput bytes (16 MiB, ~190 KB of device memory); larger
//    inputs are refused with ALPACC_E_CAPACITY;
//  * every GPU that loads the library holds one such array until the
//    process exits;
//  * all calls share the array and it keeps the last call's contents: each
//    call clears the flags it needs, so calls must not overlap on the GPU -
//    two calls in flight at once (two streams, two host threads, or two
//    handles on one device) race on it;
//  * the array's device address is looked up once per device, with that
//    device current, on the first call there (cudaGetSymbolAddress); make
//    that first call before any stream capture;
//  * every call reads the status words back and waits for the handle's
//    stream before returning, and restores the caller's current device.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/alpacc_b200.h"
#include "handle.h"
#include "kernels.h"
#include "pipeline.h"

using namespace alpacc;

namespace {

constexpr unsigned long long kNoAllocMaxInput = 16ull << 20;
constexpr unsigned long long kNoAllocTiles = (kNoAllocMaxInput + kLexData - 1) / kLexData;

// Layout of the working memory (byte offsets, 16-byte aligned pieces).
constexpr size_t kOffStatus = 0;
constexpr size_t kOffTicket = 256;
constexpr size_t kOffSt1Flag = kOffTicket + 16;
constexpr size_t kOffSt2Flag = kOffSt1Flag + ((kNoAllocTiles * 4 + 15) & ~15ull);
constexpr size_t kOffSt2Agg = kOffSt2Flag + ((kNoAllocTiles * 4 + 15) & ~15ull);
constexpr size_t kOffSt2Inc = kOffSt2Agg + kNoAllocTiles * 16;
constexpr size_t kOffSt1State = kOffSt2Inc + kNoAllocTiles * 16;
constexpr size_t kOffSt1Vec = kOffSt1State + ((kNoAllocTiles + 15) & ~15ull);
constexpr size_t kScratchBytes = kOffSt1Vec + kNoAllocTiles * 128;  // vectors of up to 128 states
static_assert(sizeof(DeviceStatus) <= kOffTicket, "status slot too small");

// The lexer's working memory for this entry point.
static __device__ __align__(256) unsigned char g_lex_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {};

// Device address of g_lex_scratch on `device` (looked up once, device current).
int scratch_address(int device, unsigned char **out) {
  if (device < 0 || device >= kMaxDevices) return ALPACC_E_INVALID;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_lex_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return ALPACC_E_CUDA;
    }
    g_scratch_addr[device] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_addr[device];
  return ALPACC_OK;
}

}  // namespace

namespace {

int lex_noalloc_on_device(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, void *d_token_ids,
                          void *d_token_starts, void *d_token_lengths, uint64_t *num_tokens);

}  // namespace

extern "C" int alpacc_gpu_lex_noalloc(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, void *d_token_ids,
                                      void *d_token_starts, void *d_token_lengths, uint64_t *num_tokens) {
  if (!g || !num_tokens || (n > 0 && (!d_in || !d_token_ids || !d_token_starts || !d_token_lengths)))
    return ALPACC_E_INVALID;
  if (g->hg.parts == ALPACC_PARTS_PARSER) return ALPACC_E_INVALID;  // tables without a lexer
  if (n > kNoAllocMaxInput) return ALPACC_E_CAPACITY;  // inputs above 16 MiB need the allocating path
  *num_tokens = 0;
  if (n == 0) return ALPACC_OK;  // lex_string accepts the empty input with no tokens
  // the caller's current device is put back on every return path
  int caller_device = -1;
  if (cudaGetDevice(&caller_device) != cudaSuccess) {
    cudaGetLastError();
    return ALPACC_E_CUDA;
  }
  if (caller_device != g->device && cudaSetDevice(g->device) != cudaSuccess) {
    cudaGetLastError();
    return ALPACC_E_CUDA;
  }
  const int rc = lex_noalloc_on_device(g, d_in, n, d_token_ids, d_token_starts, d_token_lengths, num_tokens);
  if (caller_device != g->device && cudaSetDevice(caller_device) != cudaSuccess) {
    cudaGetLastError();
    return rc < 0 ? rc : ALPACC_E_CUDA;
  }
  return rc;
}

namespace {

// The call itself, with the handle's device current.
int lex_noalloc_on_device(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, void *d_token_ids,
                          void *d_token_starts, void *d_token_lengths, uint64_t *num_tokens) {
  unsigned char *base = nullptr;
  int rc = scratch_address(g->device, &base);
  if (rc != ALPACC_OK) return rc;
  const HostGrammar &hg = g->hg;
  const LexerMachine &lm = hg.lex;
  if (lm.M > 128) return ALPACC_E_UNSUPPORTED;
  const unsigned long long tiles = (n + kLexData - 1) / kLexData;
  DeviceStatus *status = reinterpret_cast<DeviceStatus *>(base + kOffStatus);
  // clear what must start at zero: status words, ticket, look-back flags
  if (cudaMemsetAsync(base + kOffStatus, 0, kOffSt1Flag + tiles * 4, g->stream) != cudaSuccess ||
      cudaMemsetAsync(base + kOffSt2Flag, 0, tiles * 4, g->stream) != cudaSuccess) {
    cudaGetLastError();
    return ALPACC_E_CUDA;
  }
  LexArgs a = lex_args(g, d_in, n, tiles);  // the handle's tables; working memory and outputs below
  a.tok_ids = d_token_ids;
  a.tok_starts = d_token_starts;
  a.tok_lens = d_token_lengths;
  a.ticket = reinterpret_cast<unsigned *>(base + kOffTicket);
  a.st1_flag = reinterpret_cast<unsigned *>(base + kOffSt1Flag);
  a.st1_state = base + kOffSt1State;
  a.st1_vec = base + kOffSt1Vec;
  a.st2 = PairTileState{reinterpret_cast<unsigned *>(base + kOffSt2Flag),
                        reinterpret_cast<unsigned long long *>(base + kOffSt2Agg),
                        reinterpret_cast<unsigned long long *>(base + kOffSt2Inc)};
  a.status = status;
  a.diag = 0;
  const unsigned grid = (unsigned)(tiles < (unsigned long long)g->lex_grid ? tiles : (unsigned long long)g->lex_grid);
  if (launch_lex_direct(g, a, grid, g->stream) != cudaSuccess) return ALPACC_E_CUDA;
  DeviceStatus h;
  if (cudaMemcpyAsync(&h, status, sizeof h, cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
      cudaStreamSynchronize(g->stream) != cudaSuccess) {
    cudaGetLastError();
    return ALPACC_E_CUDA;
  }
  if (h.error != 0) return h.error;
  if (h.reject) return ALPACC_REJECT;
  *num_tokens = h.num_tokens;
  return ALPACC_OK;
}

}  // namespace
