// PCS opening on resident commitments: the prover side of TwoAdicFriPcs::open
// (called at vm/src/machine/prover.rs:589), each step as the Pico verifier
// checks it (vm/src/compiler/recursion/circuit/fri.rs:77-436).
//
// Device phases run on one stream; the transcript steps between them run on
// the host with the host Poseidon2 (a sponge absorbing thousands of opened
// values is sequential, and one host core runs it several times faster than
// one GPU thread):
//   1. device: 1/(z - x) tables per distinct point, opened values
//   2. host:   observe the opened values, sample alpha; alpha powers, offsets
//              and the per-point constants of every height
//   3. device: reduced openings per height, FRI commit phase (challenger on
//              the device), final element observed, proof-of-work search
//   4. host:   witness observed, query indices sampled
//   5. device: query records gathered; one read-back
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>
#include <vector>

#include "field.cuh"
#include "internal.h"
#include "open.h"
#include "runtime.h"

using namespace pico;

namespace {

constexpr uint32_t kMaxPowBits = 24;
constexpr uint32_t kSlotsPerLaunch = 4;

struct Shape {
  int field = -1;
  uint32_t log_max = 0;
  uint64_t value_words = 0;
  uint64_t query_words = 0;
  uint32_t rounds = 0;
};

pico_status check_batches(pico_ctx* ctx, const pico_open_batch* b, uint32_t n, uint32_t log_blowup, Shape& sh) {
  if (!b || n == 0) {
    set_error("open: no batches");
    return PICO_ERR_INVALID_ARG;
  }
  if (log_blowup > kLdeMaxLogBlowup) {
    set_error("open: log_blowup %u is above the supported %u", log_blowup, kLdeMaxLogBlowup);
    return PICO_ERR_INVALID_ARG;
  }
  sh = Shape{};
  for (uint32_t i = 0; i < n; i++) {
    const pico_commit* c = b[i].commit;
    if (!c || c->n_mats == 0 || (ctx && c->ctx != ctx)) {
      set_error("open: batch %u has no commitment of this context", i);
      return PICO_ERR_INVALID_ARG;
    }
    if (c->shard_log) {
      set_error("open: batch %u is one shard of a row-split commit; it holds a slice of the committed rows", i);
      return PICO_ERR_UNSUPPORTED;
    }
    if (sh.field < 0) sh.field = c->field;
    if (c->field != sh.field) {
      set_error("open: batches of different fields");
      return PICO_ERR_INVALID_ARG;
    }
    uint64_t npts = 0;
    for (uint32_t m = 0; m < c->n_mats; m++) {
      if (c->log_N[m] < log_blowup) {
        set_error("open: batch %u matrix %u has 2^%u rows, below the blowup 2^%u", i, m, c->log_N[m], log_blowup);
        return PICO_ERR_INVALID_ARG;
      }
      const uint32_t k = b[i].n_points ? b[i].n_points[m] : 0;
      npts += k;
      sh.value_words += 4ull * k * c->width[m];
      sh.query_words += c->width[m];
    }
    if (npts && !b[i].points) {
      set_error("open: batch %u has points but no point array", i);
      return PICO_ERR_INVALID_ARG;
    }
    sh.query_words += 8ull * c->log_max;
    sh.log_max = std::max(sh.log_max, c->log_max);
  }
  if (sh.log_max <= log_blowup) {
    set_error("open: tallest LDE 2^%u is not above the blowup 2^%u", sh.log_max, log_blowup);
    return PICO_ERR_INVALID_ARG;
  }
  sh.rounds = sh.log_max - log_blowup;
  for (uint32_t L = sh.log_max; L > log_blowup; L--) sh.query_words += 4 + 8ull * (L - 1);
  return PICO_OK;
}

// Device allocations of one call, released together on the stream.
struct Arena {
  cudaStream_t st = nullptr;
  std::vector<void*> ptrs;
  pico_status get(void** p, uint64_t bytes) {
    *p = nullptr;
    pico_status s = cuda_status(cudaMallocAsync(p, bytes ? bytes : 16, st), "device allocation");
    if (!s) ptrs.push_back(*p);
    return s;
  }
  template <class T>
  pico_status upload(T** dst, const std::vector<T>& v) {
    void* p;
    pico_status s = get(&p, v.size() * sizeof(T));
    if (s) return s;
    *dst = (T*)p;
    if (v.empty()) return PICO_OK;
    return cuda_status(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
  }
  void release() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
    ptrs.clear();
  }
};

// One opened (matrix, point) pair in transcript order.
struct Pair {
  uint32_t b, m, k;
  uint32_t pt;      // distinct point index
  uint64_t vofs;    // EF offset of its values
};

template <class F>
struct Opening {
  using B = Fp<F>;
  using E = Ef<F>;
  pico_ctx* ctx;
  const pico_open_batch* batches;
  uint32_t n_batches;
  uint32_t log_b;
  Shape sh;
  cudaStream_t st = nullptr;
  uint32_t slot = 0;
  Arena ar;
  uint64_t reserved = 0;
  uint32_t launches = 0;

  std::vector<Pair> pairs;
  std::vector<Ext4> pts;          // distinct points
  std::vector<uint32_t> pt_log;   // tallest LDE height each is opened at
  std::vector<uint32_t*> dtab;    // device 1/(z - x) tables

  static Ext4 ef_at(const uint32_t* p) { return Ext4{{p[0], p[1], p[2], p[3]}}; }
  static bool same(const Ext4& a, const Ext4& b) { return memcmp(a.c, b.c, 16) == 0; }
  static Ext4 ef_pow(Ext4 a, uint64_t e) {
    Ext4 r{{F::ONE, 0, 0, 0}};
    while (e) {
      if (e & 1) r = E::mul(r, a);
      a = E::mul(a, a);
      e >>= 1;
    }
    return r;
  }

  // A point on a committed coset g * H_N makes 1/(z - x) undefined (Plonky3
  // fails on the inversion); such a point is a base-field element with
  // (z / g)^N = 1.
  bool on_coset(const Ext4& z, uint32_t log_N) const {
    if (z.c[1] | z.c[2] | z.c[3]) return false;
    const uint32_t y = B::mul(z.c[0], B::inv(B::to_monty(F::GENERATOR)));
    return B::pow(y, 1ull << log_N) == F::ONE;
  }
  // the first opened point lying on its matrix's committed coset, or -1
  int64_t point_on_coset() const {
    for (size_t i = 0; i < pairs.size(); i++)
      if (on_coset(pts[pairs[i].pt], batches[pairs[i].b].commit->log_N[pairs[i].m])) return (int64_t)i;
    return -1;
  }

  void collect_points() {
    uint64_t vofs = 0;
    for (uint32_t b = 0; b < n_batches; b++) {
      const pico_commit* c = batches[b].commit;
      const uint32_t* pp = batches[b].points;
      for (uint32_t m = 0; m < c->n_mats; m++) {
        const uint32_t np = batches[b].n_points ? batches[b].n_points[m] : 0;
        for (uint32_t k = 0; k < np; k++, pp += 4) {
          const Ext4 z = ef_at(pp);
          uint32_t q = 0;
          while (q < pts.size() && !same(pts[q], z)) q++;
          if (q == pts.size()) {
            pts.push_back(z);
            pt_log.push_back(0);
          }
          pt_log[q] = std::max(pt_log[q], c->log_N[m]);
          pairs.push_back(Pair{b, m, k, q, vofs});
          vofs += c->width[m];
        }
      }
    }
  }

  // Device bytes of the reduction's S sums, their extension and its scratch
  // (heights with points; only_height < 32: that height alone).
  uint64_t reduce_bytes(uint32_t only_height = 32) const {
    uint64_t t = 0;
    for (uint32_t h = 0; h < 32; h++) {
      if (only_height < 32 && h != only_height) continue;
      std::vector<uint32_t> slots;
      for (const Pair& pr : pairs)
        if (batches[pr.b].commit->log_N[pr.m] == h && std::find(slots.begin(), slots.end(), pr.pt) == slots.end())
          slots.push_back(pr.pt);
      if (slots.empty()) continue;
      const uint64_t sw = 16ull * slots.size();  // bytes per row of S
      t += (sw << (h - log_b)) + 2 * (16ull << (h - log_b)) + (16ull << h) + (4ull << log_b) * kPwWords;
    }
    return t;
  }

  // Footprint reserved against the context budget for phase 1.
  uint64_t dtab_bytes() const {
    uint64_t s = 0;
    for (uint32_t l : pt_log) s += 16ull << (l - log_b);
    return s;
  }

  pico_status begin() {
    cudaSetDevice(ctx->device);
    st = pick_stream(ctx, nullptr, &slot);
    ar.st = st;
    return PICO_OK;
  }
  bool reserve(uint64_t bytes) {
    if (!try_reserve(ctx, bytes)) {
      set_error("open: HBM budget exceeded (%llu more bytes)", (unsigned long long)bytes);
      return false;
    }
    reserved += bytes;
    return true;
  }
  void end() {
    ar.release();
    cudaStreamSynchronize(st);
    unreserve(ctx, reserved);
    reserved = 0;
  }

  pico_status make_dtabs() {
    pico_status s;
    const TwiddleTables tw = twiddles(ctx, F::ID);
    for (size_t q = 0; q < pts.size(); q++) {
      void* p;
      // the low coset of the tallest height it is opened at: both the opened
      // values and the reduced openings are formed there
      const uint32_t lq = pt_log[q] - log_b;
      if ((s = ar.get(&p, 16ull << lq))) return s;
      dtab.push_back((uint32_t*)p);
      if ((s = cuda_status(launch_inv_denoms(F::ID, pts[q].c, lq, tw, (uint32_t*)p, st), "inverse denominators")))
        return s;
      launches++;
    }
    return PICO_OK;
  }

  // Opened values into d_values (value_words words); pairs must be collected.
  pico_status enqueue_values(uint32_t* d_values) {
    std::vector<OpenDesc> descs;
    std::vector<Ext4> scale;
    uint32_t blocks = 0, max_items = 0;
    uint64_t part = 0;
    const uint32_t g = B::to_monty(F::GENERATOR);
    for (size_t i = 0; i < pairs.size();) {
      // up to two consecutive points of the same matrix per descriptor
      const Pair& a = pairs[i];
      const pico_commit* c = batches[a.b].commit;
      const uint32_t w = c->width[a.m];
      const bool two = i + 1 < pairs.size() && pairs[i + 1].b == a.b && pairs[i + 1].m == a.m;
      const uint32_t np = two ? 2 : 1;
      if (w > 0) {
        OpenDesc d;
        memset(&d, 0, sizeof d);
        d.lde = c->lde[a.m];
        d.w = w;
        d.log_n = c->log_N[a.m] - log_b;
        // about 2^17 cells per block; at least kOpenMaxRows rows, and exactly
        // that many for matrices wider than a block of threads
        uint32_t lw = 0;
        while ((1u << lw) < w) lw++;
        d.log_rows = std::min<uint32_t>(d.log_n, w > 256 ? 10u : std::max<uint32_t>(10u, 17u - std::min(lw, 17u)));
        max_items = std::max(max_items, np * w);
        d.n_pts = np;
        d.block0 = blocks;
        d.part_off = part;
        const uint64_t n = 1ull << d.log_n;
        const uint32_t gn1 = B::pow(g, n - 1);
        const uint32_t inv_den = B::inv(B::mul(B::to_monty((uint32_t)(n % F::P)), gn1));
        const uint32_t gn = B::mul(gn1, g);
        for (uint32_t p = 0; p < 2; p++) {
          const Pair& q = pairs[i + (p < np ? p : 0)];
          d.pt[p] = q.pt;
          d.out_off[p] = q.vofs;
          Ext4 zn = ef_pow(pts[q.pt], n);
          zn.c[0] = B::sub(zn.c[0], gn);
          scale.push_back(E::scale(zn, inv_den));
        }
        const uint32_t chunks = 1u << (d.log_n - d.log_rows);
        blocks += chunks;
        part += (uint64_t)chunks * np * w;
        descs.push_back(d);
      }
      i += np;
    }
    if (descs.empty()) return PICO_OK;
    pico_status s;
    OpenDesc* d_descs;
    Ext4* d_scale;
    uint32_t** d_dt;
    void* d_part;
    if ((s = ar.upload(&d_descs, descs)) || (s = ar.upload(&d_scale, scale)) || (s = ar.upload(&d_dt, dtab)) ||
        (s = ar.get(&d_part, part * 16)))
      return s;
    if ((s = cuda_status(launch_open_values(F::ID, d_descs, (uint32_t)descs.size(), blocks, max_items, d_dt,
                                            twiddles(ctx, F::ID), (uint32_t*)d_part, (const uint32_t*)d_scale,
                                            d_values, st),
                         "opened values")))
      return s;
    launches += 2;
    return PICO_OK;
  }

  uint64_t value_cells() const {
    uint64_t v = 0;
    for (const Pair& p : pairs) {
      const pico_commit* c = batches[p.b].commit;
      v += (uint64_t)c->width[p.m] << (c->log_N[p.m] - log_b);
    }
    return v;
  }

  // Reduced openings of every height present into ro[h] (device, allocated
  // here); values are the host copy of the opened values.
  pico_status enqueue_reduce(const uint32_t* values, const Ext4& alpha, uint32_t only_height,
                             std::vector<uint32_t*>& ro, uint64_t* cells) {
    ro.assign(32, nullptr);
    pico_status s;
    // offsets per height in transcript order
    std::vector<uint64_t> num(32, 0);
    std::vector<uint32_t> off(pairs.size());
    uint32_t max_w = 1;
    for (size_t i = 0; i < pairs.size(); i++) {
      const pico_commit* c = batches[pairs[i].b].commit;
      const uint32_t h = c->log_N[pairs[i].m];
      off[i] = (uint32_t)num[h];
      num[h] += c->width[pairs[i].m];
    }
    for (uint32_t b = 0; b < n_batches; b++)
      for (uint32_t m = 0; m < batches[b].commit->n_mats; m++) max_w = std::max(max_w, batches[b].commit->width[m]);
    uint64_t T = max_w;
    for (uint64_t v : num) T = std::max(T, v);
    if (T > (1ull << 31)) {
      set_error("open: too many opened columns at one height");
      return PICO_ERR_UNSUPPORTED;
    }
    std::vector<Ext4> apow(T);
    apow[0] = Ext4{{F::ONE, 0, 0, 0}};
    for (uint64_t k = 1; k < T; k++) apow[k] = E::mul(apow[k - 1], alpha);
    // sum_j alpha^j p_j(z) per pair
    std::vector<Ext4> rys(pairs.size());
    for (size_t i = 0; i < pairs.size(); i++) {
      const uint32_t w = batches[pairs[i].b].commit->width[pairs[i].m];
      Ext4 acc{{0, 0, 0, 0}};
      for (uint32_t j = 0; j < w; j++) acc = E::add(acc, E::mul(apow[j], ef_at(values + 4 * (pairs[i].vofs + j))));
      rys[i] = acc;
    }
    Ext4* d_apow;
    if ((s = ar.upload(&d_apow, apow))) return s;
    // per height: S_z over the low coset (launches of up to kSlotsPerLaunch
    // points), its extension to the LDE domain, then the combination
    std::vector<ReduceMat> hmats;
    std::vector<ReduceTerm> hterms;
    struct Launch {
      ReduceHeight h;
      size_t mat0, n_mats, term0;
    };
    struct Height {
      uint32_t h, n_slots;
      uint32_t* s_low;     // n x 4 n_slots, natural order
      uint32_t* ro_low;    // n x 4, natural order
      size_t dinv0, k0;    // into the per-height pointer / constant arrays
    };
    std::vector<LdeMat> ext;  // ro_low -> ro[h] (N x 4, committed order), one batch
    std::vector<Launch> plan;
    std::vector<Height> heights;
    std::vector<const uint32_t*> comb_dinv;
    std::vector<Ext4> comb_k;
    std::vector<bool> present(32, false);
    for (uint32_t b = 0; b < n_batches; b++)
      for (uint32_t m = 0; m < batches[b].commit->n_mats; m++) present[batches[b].commit->log_N[m]] = true;
    uint64_t reduce_cells = 0;
    for (uint32_t h = 0; h < 32; h++) {
      if (!present[h] || (only_height < 32 && h != only_height)) continue;
      void* p;
      if ((s = ar.get(&p, 16ull << h))) return s;
      ro[h] = (uint32_t*)p;
      // distinct points at this height, in order of appearance
      std::vector<uint32_t> slots;
      for (size_t i = 0; i < pairs.size(); i++)
        if (batches[pairs[i].b].commit->log_N[pairs[i].m] == h &&
            std::find(slots.begin(), slots.end(), pairs[i].pt) == slots.end())
          slots.push_back(pairs[i].pt);
      if (slots.empty()) {
        if ((s = cuda_status(cudaMemsetAsync(p, 0, 16ull << h, st), "zero reduced opening"))) return s;
        continue;
      }
      const uint32_t log_n = h - log_b;
      const uint32_t sw = 4 * (uint32_t)slots.size();  // words per row of S
      Height H;
      memset(&H, 0, sizeof H);
      H.h = h;
      H.n_slots = (uint32_t)slots.size();
      if ((s = ar.get(&p, ((uint64_t)sw << log_n) * 4))) return s;
      H.s_low = (uint32_t*)p;
      H.dinv0 = comb_dinv.size();
      H.k0 = comb_k.size();
      for (uint32_t q : slots) comb_dinv.push_back(dtab[q]);
      comb_k.resize(comb_k.size() + slots.size(), Ext4{{0, 0, 0, 0}});
      for (size_t s0 = 0; s0 < slots.size(); s0 += kSlotsPerLaunch) {
        const size_t ns = std::min<size_t>(kSlotsPerLaunch, slots.size() - s0);
        Launch L;
        memset(&L.h, 0, sizeof L.h);
        L.h.log_h = log_n;
        L.h.n_slots = (uint32_t)ns;
        L.h.s_stride = sw;
        L.h.s_col0 = 4 * (uint32_t)s0;
        L.h.s_out = H.s_low;
        L.h.apow = reinterpret_cast<const uint4*>(d_apow);
        L.h.apow_len = (uint32_t)T;
        L.mat0 = hmats.size();
        L.term0 = hterms.size();
        // matrices of this height with a term in these slots, transcript order
        for (size_t i = 0; i < pairs.size();) {
          const Pair& a = pairs[i];
          size_t j = i;
          while (j < pairs.size() && pairs[j].b == a.b && pairs[j].m == a.m) j++;
          const pico_commit* c = batches[a.b].commit;
          if (c->log_N[a.m] == h && c->width[a.m] > 0) {
            std::vector<ReduceTerm> terms;
            for (size_t k = i; k < j; k++) {
              auto it = std::find(slots.begin() + s0, slots.begin() + s0 + ns, pairs[k].pt);
              if (it == slots.begin() + s0 + ns) continue;
              const uint32_t sl = (uint32_t)(it - (slots.begin() + s0));
              ReduceTerm T;
              memset(&T, 0, sizeof T);
              T.slot = sl;
              T.off = off[k];
              constexpr uint32_t Wm = (uint32_t)((((uint64_t)F::W) << 32) % F::P);
              for (int l = 0; l < 4; l++) {
                T.a[l] = apow[off[k]].c[l];
                T.wa[l] = l ? B::mul(T.a[l], Wm) : 0u;
              }
              terms.push_back(T);
              Ext4& K = comb_k[H.k0 + s0 + sl];
              K = E::add(K, E::mul(apow[off[k]], rys[k]));
            }
            if (!terms.empty()) {
              ReduceMat R;
              memset(&R, 0, sizeof R);
              R.lde = c->lde[a.m];
              R.w = c->width[a.m];
              R.magic = ((1ull << 32) + R.w - 1) / R.w;
              R.vec = ((uintptr_t)R.lde & 15) == 0 ? 1u : 0u;
              if (terms.size() == 1) {
                R.multi = 0;
                R.slot = terms[0].slot;
                R.off = terms[0].off;
              } else {
                R.multi = 1;
                R.n_terms = (uint32_t)terms.size();
                R.term0 = (uint32_t)(hterms.size() - L.term0);
                hterms.insert(hterms.end(), terms.begin(), terms.end());
              }
              hmats.push_back(R);
              reduce_cells += (uint64_t)R.w << log_n;
            }
          }
          i = j;
        }
        L.n_mats = hmats.size() - L.mat0;
        L.h.n_mats = (uint32_t)L.n_mats;
        plan.push_back(L);
      }
      // extension of ro from the low coset g*H_n to g*H_N: evaluations of
      // ro(g y) on H_n -> on H_N (shift 1), committed (bit-reversed) rows
      if ((s = ar.get(&p, 16ull << log_n))) return s;
      H.ro_low = (uint32_t*)p;
      LdeMat X;
      memset(&X, 0, sizeof X);
      X.log_n = log_n;
      X.log_b = log_b;
      X.w = 4;
      plan_lde_tiling(X, ctx->lde_split[F::ID][log_n]);
      X.in = H.ro_low;
      X.out = ro[h];
      if (X.log_n1) {
        if ((s = ar.get(&p, 16ull << log_n))) return s;
        X.t1 = (uint32_t*)p;
        if ((s = ar.get(&p, 16ull << h))) return s;
        X.t2 = (uint32_t*)p;
      }
      if ((s = ar.get(&p, ((uint64_t)1 << log_b) * kPwWords * 4))) return s;
      X.pw = (uint32_t*)p;
      X.shift = F::ONE;
      ext.push_back(X);
      heights.push_back(H);
    }
    ReduceMat* d_mats;
    ReduceTerm* d_terms;
    const uint32_t** d_dinv;
    Ext4* d_k;
    if ((s = ar.upload(&d_mats, hmats)) || (s = ar.upload(&d_terms, hterms)) || (s = ar.upload(&d_dinv, comb_dinv)) ||
        (s = ar.upload(&d_k, comb_k)))
      return s;
    for (Launch& L : plan) {
      L.h.mats = d_mats + L.mat0;
      L.h.terms = d_terms + L.term0;
      if ((s = cuda_status(launch_reduce(F::ID, L.h, st), "reduced opening"))) return s;
      launches++;
    }
    for (Height& H : heights) {
      if ((s = cuda_status(launch_reduce_combine(F::ID, H.h - log_b, H.s_low, 4 * H.n_slots, H.n_slots,
                                                 d_dinv + H.dinv0, reinterpret_cast<const uint32_t*>(d_k + H.k0),
                                                 H.ro_low, st),
                           "reduced opening combination")))
        return s;
      launches++;
    }
    if (!ext.empty()) {
      uint64_t nl = 0;
      if ((s = cuda_status(launch_lde(F::ID, ext.data(), (uint32_t)ext.size(), twiddles(ctx, F::ID), st, &nl),
                           "reduced opening extension")))
        return s;
      launches += (uint32_t)nl;
    }
    if (cells) *cells = reduce_cells;
    return PICO_OK;
  }
};

struct EventTimer {
  std::vector<cudaEvent_t> ev;
  pico_status mark(cudaStream_t st) {
    cudaEvent_t e;
    pico_status s = cuda_status(cudaEventCreate(&e), "event");
    if (s) return s;
    ev.push_back(e);
    return cuda_status(cudaEventRecord(e, st), "event record");
  }
  float ms(size_t a, size_t b) const {
    float t = 0;
    if (b < ev.size()) cudaEventElapsedTime(&t, ev[a], ev[b]);
    return t;
  }
  ~EventTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

pico_status open_guard_verdict() {
  GuardRecord g{};
  pico_status s = cuda_status(open_guard_fetch(&g), "guard read-back");
  if (s || !g.count) return s;
  set_error("internal bounds guard: reduction tile copies skipped %llu access(es); first: tag %llu, tile word %llu, "
            "matrix word %llu, block %llu, thread %llu",
            g.count, g.tag, g.offset, g.extent, g.block, g.thread);
  open_guard_clear();
  return PICO_ERR_CUDA;
}

template <class F>
pico_status pcs_open_t(pico_ctx* ctx, const pico_open_batch* batches, uint32_t n_batches, const Shape& sh,
                       const pico_fri_params* fp, pico_challenger* ch, uint32_t* values, uint32_t* commit_roots,
                       uint32_t* betas, uint32_t* final_poly, uint32_t* pow_witness, uint32_t* query_indices,
                       uint32_t* queries, pico_open_stats* stats) {
  using B = Fp<F>;
  const auto t0 = std::chrono::steady_clock::now();
  Opening<F> O{ctx, batches, n_batches, fp->log_blowup, sh};
  O.collect_points();
  if (O.point_on_coset() >= 0) {
    set_error("open: an opening point lies on the committed coset of its matrix");
    return PICO_ERR_INVALID_ARG;
  }
  const uint32_t log_max = sh.log_max, R = sh.rounds, nq = fp->num_queries;
  const uint64_t qw = sh.query_words;
  // footprint: tables, values, reduced openings, FRI codewords and trees, queries
  uint64_t need = O.dtab_bytes() + O.reduce_bytes() + sh.value_words * 8 + (uint64_t)nq * qw * 4 + (1u << 20);
  for (uint32_t h = 0; h <= log_max; h++) need += 16ull << h;  // reduced openings (upper bound)
  for (uint32_t r = 1; r <= R; r++) need += 16ull << (log_max - r);
  for (uint32_t r = 0; r < R; r++) need += ((2ull << (log_max - r - 1)) - 1) * 32;
  O.begin();
  if (!O.reserve(need)) return PICO_ERR_OUT_OF_MEMORY;
  EventTimer tm;
  pico_challenger tr = *ch;
  std::vector<uint32_t> final_cw(4u << fp->log_blowup);
  uint32_t best = 0xffffffffu;
  uint64_t reduce_cells = 0;
  auto run = [&]() -> pico_status {
    pico_status s;
    void* p;
    // 1. opened values
    if ((s = tm.mark(O.st))) return s;
    if ((s = O.make_dtabs())) return s;
    uint32_t* d_values = nullptr;
    if ((s = O.ar.get(&p, sh.value_words * 4))) return s;
    d_values = (uint32_t*)p;
    if ((s = O.enqueue_values(d_values))) return s;
    if ((s = tm.mark(O.st))) return s;
    if (sh.value_words &&
        (s = cuda_status(cudaMemcpyAsync(values, d_values, sh.value_words * 4, cudaMemcpyDeviceToHost, O.st),
                         "values read-back")))
      return s;
    if ((s = cuda_status(cudaStreamSynchronize(O.st), "opened values"))) return s;
    // 2. transcript: values, alpha
    for (uint64_t i = 0; i < sh.value_words; i++) host_observe(F::ID, &tr, values[i]);
    Ext4 alpha;
    for (int i = 0; i < 4; i++) alpha.c[i] = host_sample(F::ID, &tr);
    // 3. reduced openings, commit phase, proof of work
    std::vector<uint32_t*> ro;
    if ((s = tm.mark(O.st))) return s;
    if ((s = O.enqueue_reduce(values, alpha, 32, ro, &reduce_cells))) return s;
    if ((s = tm.mark(O.st))) return s;
    if ((s = cuda_status(cudaStreamSynchronize(O.st), "reduced openings"))) return s;
    std::vector<uint32_t*> cws(R + 1), trees(R);
    std::vector<const uint32_t*> inject(R, nullptr);
    cws[0] = ro[log_max];
    for (uint32_t r = 1; r <= R; r++) {
      if ((s = O.ar.get(&p, 16ull << (log_max - r)))) return s;
      cws[r] = (uint32_t*)p;
    }
    for (uint32_t r = 0; r < R; r++) {
      if ((s = O.ar.get(&p, ((2ull << (log_max - r - 1)) - 1) * 32))) return s;
      trees[r] = (uint32_t*)p;
      inject[r] = ro[log_max - r - 1];
    }
    uint32_t* d_betas;
    DevChallenger* d_ch;
    uint32_t* d_best;
    if ((s = O.ar.get(&p, 16ull * R))) return s;
    d_betas = (uint32_t*)p;
    if ((s = O.ar.get(&p, sizeof(DevChallenger)))) return s;
    d_ch = (DevChallenger*)p;
    if ((s = O.ar.get(&p, 4))) return s;
    d_best = (uint32_t*)p;
    static_assert(sizeof(DevChallenger) == sizeof(pico_challenger), "challenger layout");
    if ((s = cuda_status(cudaMemcpyAsync(d_ch, &tr, sizeof tr, cudaMemcpyHostToDevice, O.st), "challenger")))
      return s;
    uint32_t fri_launches = 0;
    if ((s = enqueue_fri_rounds(F::ID, O.st, twiddles(ctx, F::ID), log_max, R, cws, trees, d_betas, d_ch,
                                inject.data(), &fri_launches)))
      return s;
    O.launches += fri_launches;
    if ((s = cuda_status(launch_challenger_observe(F::ID, d_ch, cws[R], 4, O.st), "observe final"))) return s;
    O.launches++;
    if ((s = tm.mark(O.st))) return s;
    if ((s = cuda_status(cudaMemsetAsync(d_best, 0xff, 4, O.st), "memset"))) return s;
    // proof of work: ascending launches of 2^20 candidates; each exits at once
    // after a witness is found, so the smallest passing witness is kept
    const uint32_t chunk = 1u << 20;
    const uint32_t per_round = std::max<uint32_t>(4, (uint32_t)(((16ull << fp->proof_of_work_bits)) >> 20));
    uint64_t base = 0;
    for (;;) {
      for (uint32_t k = 0; k < per_round && base < F::P; k++, base += chunk) {
        if ((s = cuda_status(launch_grind(F::ID, d_ch, fp->proof_of_work_bits, (uint32_t)base, chunk, d_best, O.st),
                             "proof of work")))
          return s;
        O.launches++;
      }
      if ((s = cuda_status(cudaMemcpyAsync(&best, d_best, 4, cudaMemcpyDeviceToHost, O.st), "witness"))) return s;
      if ((s = cuda_status(cudaStreamSynchronize(O.st), "proof of work"))) return s;
      if (best != 0xffffffffu || base >= F::P) break;
    }
    if ((s = tm.mark(O.st))) return s;
    if (best == 0xffffffffu) {
      set_error("open: no proof-of-work witness below p");
      return PICO_ERR_INVALID_ARG;
    }
    if ((s = cuda_status(cudaMemcpyAsync(&tr, d_ch, sizeof tr, cudaMemcpyDeviceToHost, O.st), "challenger")) ||
        (s = cuda_status(cudaMemcpyAsync(final_cw.data(), cws[R], final_cw.size() * 4, cudaMemcpyDeviceToHost,
                                         O.st),
                         "final codeword")))
      return s;
    if (commit_roots)
      for (uint32_t r = 0; r < R; r++) {
        const uint64_t leaves = 1ull << (log_max - r - 1);
        if ((s = cuda_status(cudaMemcpyAsync(commit_roots + 8 * r, trees[r] + (2 * leaves - 2) * 8, 32,
                                             cudaMemcpyDeviceToHost, O.st),
                             "root copy")))
          return s;
      }
    if (betas && R &&
        (s = cuda_status(cudaMemcpyAsync(betas, d_betas, 16ull * R, cudaMemcpyDeviceToHost, O.st), "betas copy")))
      return s;
    if ((s = cuda_status(cudaStreamSynchronize(O.st), "commit phase"))) return s;
    for (size_t i = 1; i < final_cw.size() / 4; i++)
      if (memcmp(&final_cw[4 * i], &final_cw[0], 16) != 0) {
        set_error("open: final codeword is not constant (a claimed value is not the committed polynomial's)");
        return PICO_ERR_INVALID_ARG;
      }
    if (final_poly) memcpy(final_poly, final_cw.data(), 16);
    // 4. witness, query indices
    const uint32_t wm = B::to_monty(best);
    if (pow_witness) *pow_witness = wm;
    host_observe(F::ID, &tr, wm);
    (void)host_sample(F::ID, &tr);
    std::vector<uint32_t> idx(nq);
    const uint32_t mask = (uint32_t)((1ull << log_max) - 1);
    for (uint32_t q = 0; q < nq; q++) idx[q] = B::from_monty(host_sample(F::ID, &tr)) & mask;
    if (query_indices && nq) memcpy(query_indices, idx.data(), 4ull * nq);
    // 5. query records
    std::vector<QuerySeg> segs;
    uint32_t dst = 0;
    for (uint32_t b = 0; b < n_batches; b++) {
      const pico_commit* c = batches[b].commit;
      for (uint32_t m = 0; m < c->n_mats; m++) {
        if (c->width[m])
          segs.push_back(QuerySeg{c->lde[m], 0, kSegRow, log_max - c->log_N[m], c->width[m], dst});
        dst += c->width[m];
      }
      uint64_t loff = 0;
      for (uint32_t l = 0; l < c->log_max; l++) {
        segs.push_back(QuerySeg{c->layers, loff, kSegDigest, (log_max - c->log_max) + l, 0, dst});
        dst += 8;
        loff += 1ull << (c->log_max - l);
      }
    }
    for (uint32_t r = 0; r < R; r++) {
      const uint32_t L = log_max - r;
      segs.push_back(QuerySeg{cws[r], 0, kSegSibling, r, 0, dst});
      dst += 4;
      uint64_t loff = 0;
      for (uint32_t l = 0; l + 1 < L; l++) {
        segs.push_back(QuerySeg{trees[r], loff, kSegDigest, r + 1 + l, 0, dst});
        dst += 8;
        loff += 1ull << (L - 1 - l);
      }
    }
    if (dst != qw) {
      set_error("open: query record layout mismatch (%u vs %llu words)", dst, (unsigned long long)qw);
      return PICO_ERR_INVALID_ARG;
    }
    if ((s = tm.mark(O.st))) return s;
    if (nq) {
      QuerySeg* d_segs;
      uint32_t* d_idx;
      if ((s = O.ar.upload(&d_segs, segs)) || (s = O.ar.upload(&d_idx, idx))) return s;
      if ((s = O.ar.get(&p, 4ull * nq * qw))) return s;
      if ((s = cuda_status(launch_gather_queries(d_segs, (uint32_t)segs.size(), d_idx, nq, qw, (uint32_t*)p, O.st),
                           "query records")))
        return s;
      O.launches++;
      if (queries &&
          (s = cuda_status(cudaMemcpyAsync(queries, p, 4ull * nq * qw, cudaMemcpyDeviceToHost, O.st), "queries")))
        return s;
    }
    if ((s = tm.mark(O.st))) return s;
    return PICO_OK;
  };
  pico_status s = run();
  if (!s) s = guard_enqueue(ctx, O.slot, O.st);
  const cudaError_t e = cudaStreamSynchronize(O.st);
  if (!s) s = cuda_status(e, "pcs_open");  // an earlier failure keeps its own message
  if (!s) s = guard_verdict(ctx, O.slot);
  if (!s) s = open_guard_verdict();
  if (!s) *ch = tr;
  if (!s && stats) {
    memset(stats, 0, sizeof *stats);
    stats->ms_values = tm.ms(0, 1);
    stats->ms_reduce = tm.ms(2, 3);
    stats->ms_fri = tm.ms(3, 4);
    stats->ms_grind = tm.ms(4, 5);
    stats->ms_queries = tm.ms(6, 7);
    stats->value_cells = O.value_cells();
    stats->reduce_cells = reduce_cells;
    stats->launches = O.launches;
    stats->rounds = R;
  }
  O.end();
  if (!s && stats)
    stats->ms_total =
        std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return s;
}

template <class F>
pico_status open_values_t(pico_ctx* ctx, const pico_open_batch* batches, uint32_t n_batches, uint32_t log_b,
                          const Shape& sh, uint32_t* values) {
  Opening<F> O{ctx, batches, n_batches, log_b, sh};
  O.collect_points();
  if (O.point_on_coset() >= 0) {
    set_error("open_values: an opening point lies on the committed coset of its matrix");
    return PICO_ERR_INVALID_ARG;
  }
  O.begin();
  if (!O.reserve(O.dtab_bytes() + sh.value_words * 8 + (1u << 20))) return PICO_ERR_OUT_OF_MEMORY;
  auto run = [&]() -> pico_status {
    pico_status s;
    void* p;
    if ((s = O.make_dtabs())) return s;
    if ((s = O.ar.get(&p, sh.value_words * 4))) return s;
    if ((s = O.enqueue_values((uint32_t*)p))) return s;
    if (sh.value_words)
      return cuda_status(cudaMemcpyAsync(values, p, sh.value_words * 4, cudaMemcpyDeviceToHost, O.st), "values");
    return PICO_OK;
  };
  pico_status s = run();
  const cudaError_t e = cudaStreamSynchronize(O.st);
  if (!s) s = cuda_status(e, "open_values");
  O.end();
  return s;
}

template <class F>
pico_status reduced_opening_t(pico_ctx* ctx, const pico_open_batch* batches, uint32_t n_batches, uint32_t log_b,
                              const Shape& sh, const uint32_t* values, const uint32_t* alpha, uint32_t log_height,
                              uint32_t* out) {
  Opening<F> O{ctx, batches, n_batches, log_b, sh};
  O.collect_points();
  if (O.point_on_coset() >= 0) {
    set_error("reduced_opening: an opening point lies on the committed coset of its matrix");
    return PICO_ERR_INVALID_ARG;
  }
  O.begin();
  if (!O.reserve(O.dtab_bytes() + O.reduce_bytes(log_height) + (16ull << log_height) + (1u << 20)))
    return PICO_ERR_OUT_OF_MEMORY;
  auto run = [&]() -> pico_status {
    pico_status s;
    if ((s = O.make_dtabs())) return s;
    std::vector<uint32_t*> ro;
    const Ext4 a{{alpha[0], alpha[1], alpha[2], alpha[3]}};
    if ((s = O.enqueue_reduce(values, a, log_height, ro, nullptr))) return s;
    if (!ro[log_height]) {
      set_error("reduced_opening: no matrix has LDE height 2^%u", log_height);
      return PICO_ERR_INVALID_ARG;
    }
    return cuda_status(cudaMemcpyAsync(out, ro[log_height], 16ull << log_height, cudaMemcpyDeviceToHost, O.st),
                       "reduced opening");
  };
  pico_status s = run();
  if (!s) s = guard_enqueue(ctx, O.slot, O.st);
  const cudaError_t e = cudaStreamSynchronize(O.st);
  if (!s) s = cuda_status(e, "reduced_opening");
  if (!s) s = guard_verdict(ctx, O.slot);
  if (!s) s = open_guard_verdict();
  O.end();
  return s;
}

}  // namespace

extern "C" pico_status pico_gpu_open_sizes(const pico_open_batch* batches, uint32_t n_batches, uint32_t log_blowup,
                                           uint64_t* value_words, uint32_t* rounds, uint64_t* query_words) {
  Shape sh;
  pico_status s = check_batches(nullptr, batches, n_batches, log_blowup, sh);
  if (s) return s;
  if (value_words) *value_words = sh.value_words;
  if (rounds) *rounds = sh.rounds;
  if (query_words) *query_words = sh.query_words;
  return PICO_OK;
}

extern "C" pico_status pico_gpu_pcs_open(pico_ctx* ctx, const pico_open_batch* batches, uint32_t n_batches,
                                         const pico_fri_params* params, pico_challenger* ch, uint32_t* values,
                                         uint32_t* commit_roots, uint32_t* betas, uint32_t final_poly[4],
                                         uint32_t* pow_witness, uint32_t* query_indices, uint32_t* queries,
                                         pico_open_stats* stats) {
  if (!ctx || !params || !ch || !values) {
    set_error("pcs_open: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  if (ch->in_len >= 8 || ch->out_len > 8) {
    set_error("pcs_open: malformed challenger state (%u inputs, %u outputs buffered)", ch->in_len, ch->out_len);
    return PICO_ERR_INVALID_ARG;
  }
  if (params->proof_of_work_bits > kMaxPowBits) {
    set_error("pcs_open: proof_of_work_bits %u above %u", params->proof_of_work_bits, kMaxPowBits);
    return PICO_ERR_UNSUPPORTED;
  }
  if (params->num_queries && !queries && !query_indices) {
    set_error("pcs_open: no output for the queries");
    return PICO_ERR_INVALID_ARG;
  }
  Shape sh;
  pico_status s = check_batches(ctx, batches, n_batches, params->log_blowup, sh);
  if (s) return s;
  if (sh.log_max > (sh.field == PICO_KOALABEAR ? 24u : 27u)) {
    set_error("pcs_open: LDE height 2^%u above the two-adicity", sh.log_max);
    return PICO_ERR_INVALID_ARG;
  }
  if (sh.field == PICO_KOALABEAR)
    return pcs_open_t<KoalaBear>(ctx, batches, n_batches, sh, params, ch, values, commit_roots, betas, final_poly,
                                 pow_witness, query_indices, queries, stats);
  return pcs_open_t<BabyBear>(ctx, batches, n_batches, sh, params, ch, values, commit_roots, betas, final_poly,
                              pow_witness, query_indices, queries, stats);
}

extern "C" pico_status pico_gpu_open_values(pico_ctx* ctx, const pico_open_batch* batches, uint32_t n_batches,
                                            uint32_t log_blowup, uint32_t* values) {
  if (!ctx || !values) {
    set_error("open_values: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  Shape sh;
  pico_status s = check_batches(ctx, batches, n_batches, log_blowup, sh);
  if (s) return s;
  if (sh.field == PICO_KOALABEAR) return open_values_t<KoalaBear>(ctx, batches, n_batches, log_blowup, sh, values);
  return open_values_t<BabyBear>(ctx, batches, n_batches, log_blowup, sh, values);
}

extern "C" pico_status pico_gpu_reduced_opening(pico_ctx* ctx, const pico_open_batch* batches, uint32_t n_batches,
                                                uint32_t log_blowup, const uint32_t* values, const uint32_t alpha[4],
                                                uint32_t log_height, uint32_t* out) {
  if (!ctx || !alpha || !out || log_height >= 32) {
    set_error("reduced_opening: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  Shape sh;
  pico_status s = check_batches(ctx, batches, n_batches, log_blowup, sh);
  if (s) return s;
  if (sh.value_words && !values) {
    set_error("reduced_opening: values required");
    return PICO_ERR_INVALID_ARG;
  }
  if (sh.field == PICO_KOALABEAR)
    return reduced_opening_t<KoalaBear>(ctx, batches, n_batches, log_blowup, sh, values, alpha, log_height, out);
  return reduced_opening_t<BabyBear>(ctx, batches, n_batches, log_blowup, sh, values, alpha, log_height, out);
}

extern "C" pico_status pico_gpu_evaluations_on_domain(pico_ctx* ctx, const pico_commit* c, uint32_t mat_idx,
                                                      uint32_t log_domain, uint32_t* out, uint32_t flags) {
  if (!ctx || !c || c->ctx != ctx || !out || mat_idx >= c->n_mats) {
    set_error("evaluations_on_domain: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  if (c->shard_log) {
    set_error("evaluations_on_domain: the commitment is one shard of a row-split commit");
    return PICO_ERR_UNSUPPORTED;
  }
  if (log_domain > c->log_N[mat_idx]) {
    set_error("evaluations_on_domain: domain 2^%u is taller than the committed LDE 2^%u", log_domain,
              c->log_N[mat_idx]);
    return PICO_ERR_INVALID_ARG;
  }
  const uint32_t w = c->width[mat_idx];
  const uint64_t bytes = ((uint64_t)w << log_domain) * 4;
  if (bytes == 0) return PICO_OK;
  cudaSetDevice(ctx->device);
  uint32_t slot = 0;
  cudaStream_t st = pick_stream(ctx, nullptr, &slot);
  const bool dev_out = (flags & PICO_OUTPUT_DEVICE) != 0;
  if (!dev_out && !try_reserve(ctx, bytes)) {
    set_error("evaluations_on_domain: HBM budget exceeded");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  void* tmp = nullptr;
  auto run = [&]() -> pico_status {
    pico_status s;
    uint32_t* dst = out;
    if (!dev_out) {
      if ((s = cuda_status(cudaMallocAsync(&tmp, bytes, st), "device allocation"))) return s;
      dst = (uint32_t*)tmp;
    }
    if ((s = cuda_status(launch_domain_rows(c->lde[mat_idx], w, log_domain, dst, st), "domain rows"))) return s;
    if (!dev_out)
      return cuda_status(cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToHost, st), "read-back");
    return PICO_OK;
  };
  pico_status s = run();
  if (tmp) cudaFreeAsync(tmp, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (!s) s = cuda_status(e, "evaluations_on_domain");
  if (!dev_out) unreserve(ctx, bytes);
  return s;
}
