// Allocation-free coset LDE: pico_gpu_coset_lde_batch_noalloc.
//
// Some callers cannot let this library call cudaMalloc: a prover that reserves
// all of HBM for its own arena up front (so a fresh cudaMalloc fails or breaks
// its accounting), or a latency-bound loop where the device-wide
// synchronisation of cudaMalloc/cudaFree is not acceptable.  For them this
// entry point runs the same LDE kernels as pico_gpu_coset_lde_batch but takes
// its scratch (the three-pass transposes and the coset power tables) from a
// fixed array in device memory that the library declares at file scope, and
// its twiddle tables from another such array.  The caller passes device input
// and output buffers; nothing is allocated per call.
//
// Costs and rules of the static arrays:
//   - every GPU that loads this library holds kNoAllocScratchWords * 4 bytes
//     (32 MiB) plus 512 KiB of twiddle tables until the process exits;
//   - all calls share the one scratch array: calls that overlap on the GPU
//     (two streams, or two host threads) race on it and corrupt each other's
//     results; serialise them on one stream;
//   - the array keeps the previous call's contents; every word a call reads
//     is written earlier in the same call, so nothing needs clearing;
//   - the first call on a device does a one-time set-up (symbol address
//     lookup, a twiddle-fill kernel, a synchronisation) with that device
//     current; make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/pico_gpu.h"
#include "field.cuh"
#include "internal.h"
#include "runtime.h"

namespace {

// Maximum scratch: 2^b power tables of 8192 words, plus n*w + N*w words for
// the three-pass form (n > 2^11).  32 MiB = 8 Mi words.
constexpr uint64_t kNoAllocScratchWords = 8ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchWords];
// Per field: lo[j] = w^j, hi[j] = w^(j * 2^14), w of order 2^two_adicity,
// then the LDE kernels' per-stage tables.
static __device__ __align__(256) uint32_t g_noalloc_twiddles[2][2 * pico::kTwiddleWords + pico::kStageTableWords];

template <class F>
__global__ void k_fill_twiddles(uint32_t* t) {
  using B = pico::Fp<F>;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * 16384) return;
  const uint32_t w = B::pow(B::to_monty(F::GENERATOR), (uint64_t)(F::P - 1) >> F::TWO_ADICITY);
  t[i] = i < 16384 ? B::pow(w, i) : B::pow(w, (uint64_t)(i - 16384) << 14);
}

struct DeviceState {
  bool ready = false;
  uint32_t* scratch = nullptr;
  uint32_t* twiddles = nullptr;
};
std::mutex g_setup_mu;
DeviceState g_state[kMaxDevices];

// One-time set-up for the current device: host code must not use the
// symbols' names as addresses, so fetch the device addresses here.
pico_status setup_current_device(int dev, cudaStream_t st, DeviceState& out) {
  std::lock_guard<std::mutex> g(g_setup_mu);
  DeviceState& s = g_state[dev];
  if (!s.ready) {
    void* p = nullptr;
    pico_status rc = pico::cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch), "scratch symbol address");
    if (rc) return rc;
    s.scratch = (uint32_t*)p;
    rc = pico::cuda_status(cudaGetSymbolAddress(&p, g_noalloc_twiddles), "twiddle symbol address");
    if (rc) return rc;
    s.twiddles = (uint32_t*)p;
    constexpr uint32_t per_field = 2 * pico::kTwiddleWords + pico::kStageTableWords;
    k_fill_twiddles<pico::KoalaBear><<<128, 256, 0, st>>>(s.twiddles);
    k_fill_twiddles<pico::BabyBear><<<128, 256, 0, st>>>(s.twiddles + per_field);
    rc = pico::cuda_status(cudaGetLastError(), "twiddle fill");
    if (rc) return rc;
    for (int f = 0; f < 2; f++) {
      pico::TwiddleTables tt;
      tt.lo = s.twiddles + f * per_field;
      tt.hi = tt.lo + pico::kTwiddleWords;
      tt.stage = tt.lo + 2 * pico::kTwiddleWords;
      rc = pico::cuda_status(pico::launch_stage_tables(f, tt, const_cast<uint32_t*>(tt.stage), st), "stage tables");
      if (rc) return rc;
    }
    rc = pico::cuda_status(cudaStreamSynchronize(st), "twiddle fill");
    if (rc) return rc;
    s.ready = true;
  }
  out = s;
  return PICO_OK;
}

}  // namespace

extern "C" pico_status pico_gpu_coset_lde_batch_noalloc(pico_field field, const uint32_t* in, uint32_t log_n,
                                                        uint32_t width, uint32_t log_blowup, uint32_t shift,
                                                        uint32_t* out, void* stream) {
  using namespace pico;
  if ((field != PICO_KOALABEAR && field != PICO_BABYBEAR) || (!in && width) || (!out && width)) {
    set_error("coset_lde_batch_noalloc: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  const uint32_t S = field == PICO_KOALABEAR ? 24u : 27u;
  if (log_blowup > kLdeMaxLogBlowup) {
    set_error("coset_lde_batch_noalloc: log_blowup %u is above the supported %u", log_blowup, kLdeMaxLogBlowup);
    return PICO_ERR_INVALID_ARG;
  }
  if (log_n + log_blowup > S) {
    set_error("coset_lde_batch_noalloc: 2^%u rows with blowup 2^%u exceeds the two-adicity %u", log_n, log_blowup,
              S);
    return PICO_ERR_INVALID_ARG;
  }
  if (log_n > kLdeMaxLogN) {
    set_error("coset_lde_batch_noalloc: inputs above 2^%u rows are not supported", kLdeMaxLogN);
    return PICO_ERR_UNSUPPORTED;
  }
  const uint64_t n = 1ull << log_n;
  const uint64_t pw_words = (uint64_t)kPwWords << log_blowup;
  const bool three_pass = (int)log_n > kLdeSmallMaxLog;
  const uint64_t need = pw_words + (three_pass ? (uint64_t)width * (n + (n << log_blowup)) : 0);
  if (need > kNoAllocScratchWords) {
    set_error("coset_lde_batch_noalloc: this LDE needs %llu words of scratch but the static scratch holds %llu "
              "(at most 2^b*8192 + n*w*(1 + 2^b) words); use pico_gpu_coset_lde_batch",
              (unsigned long long)need, (unsigned long long)kNoAllocScratchWords);
    return PICO_ERR_INVALID_ARG;
  }
  if (width == 0) return PICO_OK;
  int dev = 0;
  pico_status rc = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("coset_lde_batch_noalloc: device %d beyond the supported %d", dev, kMaxDevices);
    return PICO_ERR_UNSUPPORTED;
  }
  cudaStream_t st = (cudaStream_t)stream;
  DeviceState ds;
  if ((rc = setup_current_device(dev, st, ds))) return rc;

  LdeMat L;
  memset(&L, 0, sizeof L);
  L.in = in;
  L.out = out;
  L.log_n = log_n;
  L.log_b = log_blowup;
  L.w = width;
  L.shift = shift % (field == PICO_KOALABEAR ? KoalaBear::P : BabyBear::P);
  L.pw = ds.scratch;
  plan_lde_tiling(L);
  if (L.log_n1) {
    L.t1 = ds.scratch + pw_words;
    L.t2 = L.t1 + (uint64_t)width * n;
  }
  TwiddleTables tw;
  tw.lo = ds.twiddles + (uint64_t)field * (2 * kTwiddleWords + kStageTableWords);
  tw.hi = tw.lo + kTwiddleWords;
  tw.stage = tw.lo + 2 * kTwiddleWords;
  return cuda_status(launch_lde(field, &L, 1, tw, st), "coset_lde_batch_noalloc launch");
}

// Bounds-guard verdict of the allocation-free LDE.  Its kernels record a
// skipped out-of-range access in the LDE unit's device record instead of
// making it; the call itself is asynchronous and cannot report that, so the
// caller asks here after its stream has reached the call.  This reads the
// record into host memory (nothing is allocated) and clears it.
extern "C" pico_status pico_gpu_noalloc_status(void* stream) {
  using namespace pico;
  pico_status rc = cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "noalloc_status: stream");
  if (rc) return rc;
  GuardRecord g{};
  if ((rc = cuda_status(lde_guard_fetch(&g, (cudaStream_t)stream), "noalloc_status: guard read-back"))) return rc;
  if ((rc = cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "noalloc_status: guard read-back"))) return rc;
  if (!g.count) return PICO_OK;
  set_error("internal bounds guard: LDE kernel skipped %llu access(es); first: tag %llu, offset %llu of %llu, "
            "block %llu, thread %llu",
            g.count, g.tag, g.offset, g.extent, g.block, g.thread);
  lde_guard_clear();
  return PICO_ERR_CUDA;
}
