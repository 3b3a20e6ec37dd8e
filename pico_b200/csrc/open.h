// Device-side descriptors and launchers of the PCS opening (open_kernels.cu),
// shared with the host orchestration (open_host.cu).  Not part of the ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pico_gpu.h"
#include "field.cuh"
#include "internal.h"

namespace pico {

constexpr uint32_t kOpenMaxRows = 1024;  // low-coset rows whose weights k_open_partial holds in shared memory

// One matrix of the opened-values pass and up to two of its points.
struct OpenDesc {
  const uint32_t* lde;  // committed LDE, bit-reversed rows, row-major
  uint32_t w;
  uint32_t log_n;       // low coset (trace) height
  uint32_t log_rows;    // rows per block (at most log2(kOpenMaxRows) when w > 256)
  uint32_t n_pts;       // 1 or 2
  uint32_t pt[2];       // distinct-point index of each point (its 1/(z - x) table)
  uint32_t block0;      // first block of this descriptor
  uint32_t pad;
  uint64_t part_off;    // EF offset of this descriptor's partial sums
  uint64_t out_off[2];  // EF offset of each point's values in the output
};

// Reduced opening of one height.
struct ReduceMat {
  const uint32_t* lde;
  uint64_t magic;    // ceil(2^32 / w): f / w = (f * magic) >> 32 for f < 32 w, w <= 32
  uint32_t w;
  uint32_t multi;    // 0: one point (slot, off); 1: n_terms terms from term0
  uint32_t slot, off;
  uint32_t n_terms, term0;
  uint32_t vec;      // the matrix starts 16-byte aligned (16-byte copies where rows allow)
  uint32_t pad;
};
// One (point, alpha^off) term of a matrix opened at several points: a = alpha^off
// and W a (entries 1..3), Monty form.
struct ReduceTerm {
  uint32_t slot, off;
  uint32_t a[4];
  uint32_t wa[4];
};
// One launch of k_reduce: the low coset (2^log_h rows) of the matrices of one
// height, for up to four of its points; writes S_q (EF4) for each at row
// rev(i) of s_out, columns s_col0 + 4q .. + 3 (rows of s_stride words).
struct ReduceHeight {
  uint32_t log_h;        // rows of the low coset (log)
  uint32_t n_mats;
  uint32_t n_slots;      // points handled by this launch (1..4)
  uint32_t s_stride;
  uint32_t s_col0;
  uint32_t apow_len;
  const ReduceMat* mats;
  const ReduceTerm* terms;
  const uint4* apow;     // alpha^k, EF4, k < apow_len
  uint32_t* s_out;
};

// Pieces of a query record.
enum : uint32_t { kSegRow = 0, kSegDigest = 1, kSegSibling = 2 };
struct QuerySeg {
  const uint32_t* base;
  uint64_t level_off;  // kSegDigest: digests before this layer
  uint32_t kind;
  uint32_t shift;      // the record uses (index >> shift)
  uint32_t width;      // kSegRow: row width
  uint32_t dst;        // word offset in the record
};

cudaError_t launch_inv_denoms(int field, const uint32_t z[4], uint32_t log_h, TwiddleTables tw, uint32_t* out,
                              cudaStream_t st);
// max_items: the largest n_pts * w of the descriptors (finalize grid width).
cudaError_t launch_open_values(int field, const OpenDesc* descs, uint32_t n_desc, uint32_t n_blocks,
                               uint32_t max_items, const uint32_t* const* dinv_tables, TwiddleTables tw,
                               uint32_t* partial, const uint32_t* scale, uint32_t* values, cudaStream_t st);
cudaError_t launch_reduce(int field, const ReduceHeight& h, cudaStream_t st);
// ro[k] = sum_q dinv[q][rev(k)] * (K[q] - S[k][q]) for k < 2^log_n, natural order
// (S rows of s_stride words).
cudaError_t launch_reduce_combine(int field, uint32_t log_n, const uint32_t* s, uint32_t s_stride, uint32_t n_slots,
                                  const uint32_t* const* dinv, const uint32_t* K, uint32_t* ro, cudaStream_t st);
// Bounds guard of the reduction's tile copies (synchronous read-back / clear).
cudaError_t open_guard_fetch(GuardRecord* dst);
cudaError_t open_guard_clear();
// out row k = lde row rev(k), k < 2^log_d (rows of w words)
cudaError_t launch_domain_rows(const uint32_t* lde, uint32_t w, uint32_t log_d, uint32_t* out, cudaStream_t st);
cudaError_t launch_gather_queries(const QuerySeg* segs, uint32_t n_segs, const uint32_t* indices, uint32_t n_queries,
                                  uint64_t query_words, uint32_t* out, cudaStream_t st);

// p2_kernels.cu: smallest witness in [base, base + count) whose observation
// makes the challenger's next sample have `bits` low zero bits; atomicMin into
// *best (left unchanged when none; blocks exit early once *best is set).
cudaError_t launch_grind(int field, const DevChallenger* ch, uint32_t bits, uint32_t base, uint32_t count,
                         uint32_t* best, cudaStream_t st);

// Host Poseidon2 and duplex challenger (api.cu), for transcript steps that
// run on the host between device phases.
void host_permute(int field, uint32_t s[16]);
void host_observe(int field, pico_challenger* ch, uint32_t v);
uint32_t host_sample(int field, pico_challenger* ch);

}  // namespace pico
