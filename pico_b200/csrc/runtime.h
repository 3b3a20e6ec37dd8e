// Host runtime shared by the C-ABI translation units: context, device memory,
// commit planning and enqueueing.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pico_gpu.h"
#include "internal.h"

namespace pico {

void set_error(const char* fmt, ...);
pico_status cuda_status(cudaError_t e, const char* what);

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

// One matrix of a commit after planning.
struct PlannedMat {
  uint32_t input_idx;  // position in the caller's array
  uint32_t log_n;      // trace height (log)
  uint32_t log_N;      // committed (LDE) height (log)
  uint32_t w;
  uint32_t shift;      // Monty
  const uint32_t* src; // caller's input pointer (host or device)
};

struct CommitPlan {
  int field = 0;
  uint32_t log_b = 0;
  bool extend = true;            // false: mmcs_commit of already-extended matrices
  bool input_device = false;
  bool plain = false;
  bool wide_groups = false;      // a height group has more matrices with columns than kMaxSegs
  std::vector<PlannedMat> mats;  // in commit order (stable, tallest first)
  // height groups in commit order: [begin, end) into mats
  std::vector<std::pair<uint32_t, uint32_t>> groups;
  uint32_t log_max = 0;
  // One shard of a commit split by rows over 2^shard_log devices: every LDE
  // computes only its rows [shard N / 2^k, (shard + 1) N / 2^k) (k <= log_b),
  // and log_N / log_max count the shard's rows.
  uint32_t shard_log = 0, shard = 0;
  uint64_t bytes_resident = 0;   // LDEs + digest layers
  uint64_t bytes_scratch = 0;    // input copies, NTT scratch, tables
  uint64_t cells = 0;            // sum of trace cells
  uint64_t lde_cells = 0;
  uint64_t permutations = 0;     // tree permutations
  uint64_t leaf_permutations = 0;
};

pico_status plan_commit(int field, const pico_matrix* mats, uint32_t n, uint32_t log_b, uint32_t flags, bool extend,
                        CommitPlan& plan, uint32_t shard_log = 0, uint32_t shard = 0);

struct Server;  // serving.h
constexpr uint32_t kMaxGroup = 16;     // serving: largest group of requests sharing launches
constexpr uint32_t kDefaultGroup = 8;  // pico_config.max_group = 0

// Stream-ordered device allocation of the library (failure injection for
// tests included); free with cudaFreeAsync on a stream ordered after st.
pico_status device_alloc(void** p, size_t bytes, cudaStream_t st);
bool try_reserve(pico_ctx* ctx, uint64_t bytes);
void unreserve(pico_ctx* ctx, uint64_t bytes);
cudaStream_t pick_stream(pico_ctx* ctx, cudaStream_t* copy_stream = nullptr, uint32_t* slot = nullptr);
cudaStream_t aux_stream(pico_ctx* ctx);
TwiddleTables twiddles(pico_ctx* ctx, int field);
pico_status enqueue_commit(pico_ctx* ctx, const CommitPlan& plan, cudaStream_t st, cudaStream_t cst,
                           pico_commit* c, std::vector<void*>& scratch, uint32_t* root_host);
// Several extended, batched commits of device inputs of one field on st,
// sharing their LDE and row-hashing launches (serving admits them together).
pico_status enqueue_commit_group(pico_ctx* ctx, const std::vector<const CommitPlan*>& plans, cudaStream_t st,
                                 const std::vector<pico_commit*>& commits, std::vector<void*>& scratch,
                                 const std::vector<uint32_t*>& root_host);
void free_commit_buffers(pico_commit* c, cudaStream_t st);
// Bounds guards of the kernels (GuardRecord): guard_enqueue copies both
// units' records into the slot's pinned host records on st; after st has
// been synchronised, guard_verdict returns PICO_OK, or an error naming the
// first skipped access (and clears the device records).
// FRI commit-phase rounds on st (fri_host.cu): round r's tree over
// codewords[r] viewed as a (len/2) x 8 matrix goes into trees[r] (the leaves of
// round 0 hashed first, those of later rounds by the previous fold), its root
// is observed and beta sampled into d_betas[r] by the device challenger (d_ch
// null: d_betas holds the challenges already), and the fold writes
// codewords[r + 1], adding inject[r] when that is non-null.  *launches counts
// the kernels.
pico_status enqueue_fri_rounds(int field, cudaStream_t st, const TwiddleTables& tw, uint32_t log_n, uint32_t R,
                               const std::vector<uint32_t*>& codewords, const std::vector<uint32_t*>& trees,
                               uint32_t* d_betas, DevChallenger* d_ch, const uint32_t* const* inject,
                               uint32_t* launches = nullptr);
pico_status guard_enqueue(pico_ctx* ctx, uint32_t slot, cudaStream_t st);
pico_status guard_verdict(pico_ctx* ctx, uint32_t slot, std::string* msg = nullptr);
pico_status finish_stats(pico_commit* c);
// One JSON line per finished commit or served request into the file named by
// PICO_METRICS_LOG (nothing when unset); queued_us < 0 for synchronous commits;
// `group`: members of the group a served request was admitted in.
void metrics_record(const char* kind, int field, uint32_t n_mats, uint32_t log_b, uint32_t flags,
                    const pico_commit_stats& st, double queued_us, double run_us, uint32_t group = 0);

}  // namespace pico

struct pico_ctx {
  int device = 0;
  int sm_count = 0;
  uint64_t budget = 0;
  uint64_t reserved = 0;
  std::mutex mu;               // guards budget accounting
  std::condition_variable cv;  // signalled whenever reserved memory is returned
  std::vector<cudaStream_t> streams;
  std::vector<cudaStream_t> copy_streams;  // paired with streams[i]: host -> device input copies
  std::atomic<uint32_t> next_stream{0};
  std::vector<cudaStream_t> aux_streams;  // read-backs and releases of finished work
  std::atomic<uint32_t> next_aux{0};
  uint32_t* tw[2] = {nullptr, nullptr};  // per-field twiddle tables (lo | hi | stage)
  pico::GuardRecord* guard_host = nullptr;  // pinned: 2 records (LDE, hashing) per stream slot
  pico::Server* server = nullptr;
  uint32_t max_inflight = 0;  // serving: requests on the device at once
  uint32_t max_group = pico::kDefaultGroup;  // serving: requests admitted together into one slot (shared launches)
  // Autotuned choices (pico_gpu_autotune), per field: the LDE's four-step
  // split log2 n1 per height (0 = default) and the row-hashing block size.
  uint8_t lde_split[2][pico::kLdeMaxLogN + 1] = {};
  uint32_t hash_block[2] = {256, 256};
  ~pico_ctx();
};

// Opaque public handles.
struct pico_commit {
  pico_ctx* ctx = nullptr;
  int field = 0;
  uint32_t log_max = 0;
  uint32_t n_mats = 0;
  std::vector<uint32_t*> lde;     // per input index: device LDE (bit-reversed rows)
  std::vector<uint32_t> log_N;    // per input index
  std::vector<uint32_t> width;    // per input index
  std::vector<void*> blocks;      // the commit's device allocations: owned LDEs / copied inputs, layers
  uint32_t* layers = nullptr;     // all digest layers, leaves first (in one of the blocks)
  uint32_t shard_log = 0;         // > 0: one shard of a row-split commit (pico_gpu_commit_shard)
  uint64_t bytes_resident = 0;
  uint32_t root[8] = {0};
  // events (see finish_stats): compute-stream phases 0, 3, 4, copy stream 5..6,
  // and a pair around each LDE and each row-hashing launch
  cudaEvent_t ev[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  enum PhaseKind { kLde = 0, kLeaves = 1, kRows = 2 };
  struct Phase {
    int kind = kLde;
    cudaEvent_t begin = nullptr, end = nullptr;
  };
  std::vector<Phase> phases;
  void destroy_events();
  pico_commit_stats stats{};
  ~pico_commit();
};

struct pico_fri {
  pico_ctx* ctx = nullptr;
  int field = 0;
  uint32_t log_n = 0, rounds = 0;
  std::vector<uint32_t*> codewords;  // round r: 2^(log_n - r) x 4
  std::vector<uint32_t*> trees;      // round r: digest layers over 2^(log_n - r - 1) leaves
  void* arena = nullptr;             // codewords and trees are views into it
  uint64_t bytes_resident = 0;
};
