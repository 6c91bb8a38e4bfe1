// Shared device utilities of the sm_100a solve path.
#pragma once

#include <cuda_runtime.h>
#include <cuda/atomic>
#include <cstdint>
#include <type_traits>

#include "sfr3d_b200.h"

namespace sfr {

constexpr int kWarp = 32;

// ----------------------------------------------------------------------
// Loads.  The matrix is read once per sweep: streaming (evict-first) loads
// keep it from pushing the Krylov vectors out of L2.
// Vectors that other blocks of the same launch write (persistent kernels,
// block partials) are read with plain (weak, L1-cached) loads, only after a
// synchronisation that orders the writes before them: the grid barrier (the
// writer's bar.sync + device-scope release, the reader's device-scope
// acquire + bar.sync) or the last-block fence/atomic/fence pattern.  Under
// the PTX memory model those reads observe the writes; the device-scope
// acquire is what discards stale L1 lines.  Never ld.global.nc for them: the
// non-coherent path is outside that guarantee.
// ----------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T ld_stream(const T *p) { return __ldcs(p); }
template <typename T>
__device__ __forceinline__ T ld_vec(const T *p) { return *p; }
template <typename T>
__device__ __forceinline__ void st_vec(T *p, T v) { __stcg(p, v); }
// Data no thread writes while the kernel runs: a plain (L1-cached, LSU) load.
// Neighbouring rows of a warp share most of their gathers, and for divergent
// gathers the LSU path sustains far more requests than the non-coherent
// read-only path (ld.global.nc).
template <typename T>
__device__ __forceinline__ T ld_ro(const T *p) { return *p; }

// ----------------------------------------------------------------------
// Arithmetic that rounds exactly as the reference's host code does (one
// rounding per multiply and per add; no FMA contraction).  Used by the FP64
// path so that every SpMV row and vector update is bit-identical to
// HccaBlas.c / Cg.c / Bicgstab.c.
// ----------------------------------------------------------------------
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
// IEEE division and square root, correctly rounded (what the host's / and
// sqrt give)
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }

// ----------------------------------------------------------------------
// Deterministic reductions: fixed shuffle tree inside a warp, fixed tree
// over the warps of a block, fixed sequential+tree order over the blocks.
// ----------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;  // valid in lane 0
}

// Reduce NV per-thread values over the block; thread 0 writes
// part[v * stride + blockIdx.x].  `sm` holds NV * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_partials(const double (&acc)[NV], double *part,
                                               int stride, double *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double w = warp_sum(acc[v]);
    if (lane == 0) sm[v * 32 + warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double w = lane < nwarps ? sm[v * 32 + lane] : 0.0;
      w = warp_sum(w);
      if (lane == 0) st_vec(part + v * stride + blockIdx.x, w);
    }
  }
  __syncthreads();
}

// Every block sums the nblocks partials of each value in the same order, so
// all blocks hold bit-identical totals.  Result broadcast through `sm`.
template <int NV>
__device__ __forceinline__ void grid_totals(const double *part, int stride, int nblocks,
                                            double (&out)[NV], double *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = 0.0;
      for (int b = lane; b < nblocks; b += 32) s += ld_vec(part + v * stride + b);
      s = warp_sum(s);
      if (lane == 0) sm[v] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v] = sm[v];
  __syncthreads();
}

// ----------------------------------------------------------------------
// Grid-wide barrier for a cooperative (co-resident) launch.  Every wait is
// bounded: after `spin_limit` polls the block records SFR_TIMEOUT in *err and
// returns false; a block that sees *err set stops waiting at once, so every
// block leaves the kernel in bounded time.
// ----------------------------------------------------------------------
struct GridSync {
  unsigned int *count;
  unsigned int *gen;
  int *err;
  unsigned int nblocks;
  unsigned int spin_limit;
};

__device__ __forceinline__ bool grid_sync(const GridSync &g) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(*g.gen);
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(*g.count);
    cuda::atomic_ref<int, cuda::thread_scope_device> err(*g.err);
    int ok = 1;
    const unsigned int my = gen.load(cuda::memory_order_relaxed);
    const unsigned int prev = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
    if (prev == g.nblocks - 1) {
      cnt.store(0u, cuda::memory_order_relaxed);
      gen.store(my + 1u, cuda::memory_order_release);
    } else {
      unsigned int spins = 0;
      while (gen.load(cuda::memory_order_acquire) == my) {
        if (err.load(cuda::memory_order_relaxed) != 0) { ok = 0; break; }
        if (++spins > g.spin_limit) {
          int expected = 0;
          err.compare_exchange_strong(expected, SFR_TIMEOUT, cuda::memory_order_relaxed);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    if (ok && err.load(cuda::memory_order_relaxed) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ----------------------------------------------------------------------
// Wait on the blocks a phase gathers from.  A block whose next phase reads a
// vector only at its rows' columns needs the updates of the blocks owning
// those columns -- for a banded (RCM-ordered) matrix a few neighbouring
// blocks -- not of the whole grid.  Each block publishes the number of
// updates it has finished in its own 64-byte slot of `ticks` (16 words a
// block, zero at launch; release) and polls the slots of blocks [lo, hi]
// (acquire; thread t watches block lo + t, so hi - lo < blockDim.x).  The
// caller keeps the blocks from rewriting the vector while another still
// reads it (a global exchange between the reads and the next writes).
// Bounded: after spin_limit polls a block records SFR_TIMEOUT in *err; a
// block that sees *err set stops waiting.  Returns false on either.
// ----------------------------------------------------------------------
__device__ __forceinline__ bool neighbour_wait(unsigned *ticks, int *err_word,
                                               unsigned spin_limit, unsigned tick, int lo,
                                               int hi) {
  __syncthreads();  // the block's writes come before the release
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device>(ticks[16 * blockIdx.x])
        .store(tick, cuda::memory_order_release);
  }
  const int t = lo + static_cast<int>(threadIdx.x);
  const bool watcher = t <= hi && t != static_cast<int>(blockIdx.x);
  int seen = !watcher;
  int ok = 1;
  cuda::atomic_ref<int, cuda::thread_scope_device> err(*err_word);
  for (unsigned spins = 0;; ++spins) {
    if (!seen)
      seen = cuda::atomic_ref<unsigned, cuda::thread_scope_device>(ticks[16 * t])
                 .load(cuda::memory_order_acquire) >= tick;
    if (__syncthreads_and(seen)) break;
    if ((spins & 63u) == 63u &&
        __syncthreads_or(threadIdx.x == 0 && err.load(cuda::memory_order_relaxed) != 0)) {
      ok = 0;
      break;
    }
    if (spins > spin_limit) {
      if (threadIdx.x == 0) {
        int expected = 0;
        err.compare_exchange_strong(expected, SFR_TIMEOUT, cuda::memory_order_relaxed);
      }
      ok = 0;
      break;
    }
  }
  return ok != 0;
}

// The block owning row `row` under block_slices's partition of nslices
// slices over gridDim.x blocks.
__device__ __forceinline__ int owner_block(int row, int nslices) {
  const long long G = gridDim.x, ns = nslices, sl = row / 32;
  return static_cast<int>(((sl + 1) * G + ns - 1) / ns - 1);
}

// ----------------------------------------------------------------------
// Sliced ELLPACK (SELL-32) view.  Rows are grouped in slices of 32; slice s
// holds w_s = (sptr[s+1]-sptr[s])/32 slots, stored slot-major so that lane l
// of a warp reads row 32s+l.  Slot k of a row is its k-th off-diagonal in the
// reference's summation order; the diagonal is separate and summed first.
// Padded slots have col = row and val = 0.
// ----------------------------------------------------------------------
template <typename V>
struct SellView {
  int n;
  int nslices;
  const int *sptr;
  const int *col;
  const V *val;
  const V *diag;
};

// Row r = 32*s + lane of A*x with the reference's rounding: diagonal product
// first, then each slot's product added in order.
template <typename V, typename XV>
__device__ __forceinline__ double row_spmv_exact(const SellView<V> &A, int s, int lane,
                                                 const XV *x) {
  const int r = s * kWarp + lane;
  const int base = __ldg(A.sptr + s);
  const int w = (__ldg(A.sptr + s + 1) - base) >> 5;
  double t = xmul(static_cast<double>(ld_stream(A.diag + r)), static_cast<double>(ld_vec(x + r)));
  const int *c = A.col + base + lane;
  const V *v = A.val + base + lane;
#pragma unroll 4
  for (int k = 0; k < w; ++k) {
    const int j = ld_stream(c + k * kWarp);
    const double a = static_cast<double>(ld_stream(v + k * kWarp));
    t = xadd(t, xmul(a, static_cast<double>(ld_vec(x + j))));
  }
  return t;
}

// Column of a slot: an absolute index (int), or a 16-bit offset from the
// row (int16_t: patterns whose bandwidth is below 32768, 2 bytes a slot
// instead of 4).
__device__ __forceinline__ int slot_col(const int *c, int k, int) { return ld_stream(c + k); }
__device__ __forceinline__ int slot_col(const int16_t *c, int k, int row) {
  return row + static_cast<int>(ld_stream(c + k));
}

// The columns of a SELL matrix's slots: offsets when the pattern has them,
// else absolute indices.
struct SlotCols {
  const int *col;
  const int16_t *off;  // null when the bandwidth does not fit 16 bits
};

// The slot columns a kernel instantiation reads: 16-bit offsets (I =
// int16_t) or absolute indices (I = int).  Separate instantiations keep each
// SpMV phase at the register count of one index form.
template <typename I>
__device__ __forceinline__ const I *cols_of(const SlotCols &c);
template <>
__device__ __forceinline__ const int *cols_of<int>(const SlotCols &c) { return c.col; }
template <>
__device__ __forceinline__ const int16_t *cols_of<int16_t>(const SlotCols &c) { return c.off; }

// y_k[row] = diag*v(row) + sum_e val_e * v(col_e) for K vectors given by a
// gather functor g(k, col), accumulated in Acc: exact FP64 (kExact: the
// reference's rounding, one rounding per product and per sum), or with FMA.
// Values may be FP32 with FP64 accumulation (the mixed path).  A row's column
// indices and values are loaded six at a time before any gather, so all of
// them are in flight together.
template <int K, typename Acc, bool kExact, typename V, typename DV, typename G,
          typename I = int>
__device__ __forceinline__ void row_product_t(const int *sptr, const I *colp, const V *valp,
                                              const DV *const *diagp, int s, int lane,
                                              const int (&act)[K], G g, Acc (&y)[K]) {
  const int row = s * kWarp + lane;
  const int base = __ldg(sptr + s);
  const int w = (__ldg(sptr + s + 1) - base) >> 5;
  const I *c = colp + base + lane;
  const V *v = valp + base + lane;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (act[k]) {
      const Acc dv = static_cast<Acc>(ld_vec(diagp[k] + row));
      const Acc gv = static_cast<Acc>(g(k, row));
      y[k] = kExact ? xmul(dv, gv) : dv * gv;
    }
  for (int e0 = 0; e0 < w; e0 += 6) {
    int jj[6];
    Acc vv[6];
#pragma unroll
    for (int u = 0; u < 6; ++u)
      if (e0 + u < w) {
        jj[u] = slot_col(c, (e0 + u) * kWarp, row);
        vv[u] = static_cast<Acc>(ld_stream(v + (e0 + u) * kWarp));
      }
#pragma unroll
    for (int u = 0; u < 6; ++u)
      if (e0 + u < w) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          if (act[k]) {
            const Acc gv = static_cast<Acc>(g(k, jj[u]));
            y[k] = kExact ? xadd(y[k], xmul(vv[u], gv)) : fma(vv[u], gv, y[k]);
          }
      }
  }
}

// L2 prefetch for an iteration's SpMV phase: lane 0 of each warp asks for
// the slice the warp reaches `pf` rounds later (a round: every warp of the
// block one slice further), within the block's own slices.  A slice's slot
// columns and values are each one contiguous run (slot-major, 32 rows a
// slot), so one bulk prefetch covers each: values at 256 B (FP64) / 128 B
// (FP32) and columns at 64 B boundaries, sizes multiples of 64 B -- both
// within cp.async.bulk's 16-byte rule.
template <typename I, typename V>
__device__ __forceinline__ void prefetch_slice_ahead(int pf, const int *sptr, const I *cols,
                                                     const V *vals, int s, int s1) {
  if (pf <= 0 || (threadIdx.x & 31) != 0) return;
  const int t = s + pf * static_cast<int>(blockDim.x >> 5);
  if (t >= s1) return;
  const int b = __ldg(sptr + t);
  const int e = __ldg(sptr + t + 1);
  if (e <= b) return;
  const unsigned nv = static_cast<unsigned>(e - b) * sizeof(V);
  const unsigned nc = static_cast<unsigned>(e - b) * sizeof(I);
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(vals + b), "r"(nv) : "memory");
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(cols + b), "r"(nc) : "memory");
}

// A warp's slices s0 + warp, s0 + warp + warps, ... (< s1) of a K-vector
// SpMV phase, with the loads of each slice ordered for latency: the next
// slice's extent is read one slice ahead, and every load that does not
// depend on a column index -- the row's own operands of the phase (pre(k,
// row), e.g. r and r0 for a dot), the diagonal and each vector at the row --
// is issued with the slot columns and values, before the first gather.  A
// slice then costs two dependent memory round trips (columns, then gathers)
// instead of four.  The arithmetic is row_product_t's: diagonal product
// first, then each slot's product in order.  post(k, row, y_k, pre_k) runs
// for each active k of every row below n.  pf: prefetch_slice_ahead's
// distance (0: off).
template <int K, typename Acc, bool kExact, typename V, typename DV, typename I, typename G,
          typename Pre, typename Post>
__device__ __forceinline__ void slice_rows(int n, const int *sptr, const I *colp,
                                           const V *valp, const DV *const *diagp, int s0,
                                           int s1, int pf, const int (&act)[K], G g, Pre pre,
                                           Post post) {
  using E = decltype(pre(0, 0));
  const int lane = threadIdx.x & 31;
  const int step = static_cast<int>(blockDim.x >> 5);
  int s = s0 + static_cast<int>(threadIdx.x >> 5);
  if (s >= s1) return;
  int base = __ldg(sptr + s), end = __ldg(sptr + s + 1);
  for (; s < s1; s += step) {
    prefetch_slice_ahead(pf, sptr, colp, valp, s, s1);
    const int row = s * kWarp + lane;
    int nbase = 0, nend = 0;
    if (s + step < s1) {
      nbase = __ldg(sptr + s + step);
      nend = __ldg(sptr + s + step + 1);
    }
    if (row < n) {
      E ex[K];
      Acc y[K], dv[K], gv[K];
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (act[k]) {
          ex[k] = pre(k, row);
          dv[k] = static_cast<Acc>(ld_vec(diagp[k] + row));
          gv[k] = static_cast<Acc>(g(k, row));
        }
      const int w = (end - base) >> 5;
      const I *c = colp + base + lane;
      const V *v = valp + base + lane;
      int jj[6];
      Acc vv[6];
#pragma unroll
      for (int u = 0; u < 6; ++u)
        if (u < w) {
          jj[u] = slot_col(c, u * kWarp, row);
          vv[u] = static_cast<Acc>(ld_stream(v + u * kWarp));
        }
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (act[k]) y[k] = kExact ? xmul(dv[k], gv[k]) : dv[k] * gv[k];
      for (int e0 = 0; e0 < w; e0 += 6) {
        if (e0 > 0) {
#pragma unroll
          for (int u = 0; u < 6; ++u)
            if (e0 + u < w) {
              jj[u] = slot_col(c, (e0 + u) * kWarp, row);
              vv[u] = static_cast<Acc>(ld_stream(v + (e0 + u) * kWarp));
            }
        }
#pragma unroll
        for (int u = 0; u < 6; ++u)
          if (e0 + u < w) {
#pragma unroll
            for (int k = 0; k < K; ++k)
              if (act[k]) {
                const Acc t = static_cast<Acc>(g(k, jj[u]));
                y[k] = kExact ? xadd(y[k], xmul(vv[u], t)) : fma(vv[u], t, y[k]);
              }
          }
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (act[k]) post(k, row, y[k], ex[k]);
    }
    base = nbase;
    end = nend;
  }
}

// ----------------------------------------------------------------------
// Slices staged in shared memory by the bulk-copy (TMA) engine.
//
// A slice's slot values and slot columns are each one contiguous run
// (slot-major, 32 rows a slot) that starts at sptr[s], a multiple of 32
// elements: 128 B for FP32 values, 256 B for FP64, 64 B for 16-bit columns,
// so both copies start and end on 16-byte boundaries as cp.async.bulk
// requires (the arrays themselves are cudaMalloc'd, 256-byte aligned).
// Each warp owns kStages stage buffers with one mbarrier each; lane 0
// copies the warp's slice kStages slices ahead into a free stage, and the
// warp reads the slice from shared memory once that stage's mbarrier phase
// completes.  The matrix stream then runs behind the warp's arithmetic, and
// only the gathers wait on memory.  No multicast, no tensor map.
// ----------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
// Order this thread's mbarrier inits and generic-proxy accesses of shared
// memory before later async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Column of a staged slot (shared memory): absolute, or row + offset.
__device__ __forceinline__ int smem_col(const int *c, int k, int) { return c[k]; }
__device__ __forceinline__ int smem_col(const int16_t *c, int k, int row) {
  return row + static_cast<int>(c[k]);
}

// Bytes of one warp's stages: kStages mbarriers (padded to 16 bytes), then
// kStages value buffers, then kStages column buffers of `cap` slots each
// (cap a multiple of 32).
template <typename V, typename I, int kStages>
__host__ __device__ constexpr int staged_warp_bytes(int cap) {
  return ((kStages * 8 + 15) / 16) * 16 + kStages * cap * static_cast<int>(sizeof(V) + sizeof(I));
}

// slice_rows with the slices staged in shared memory (`smem`: the block's
// dynamic shared memory, staged_warp_bytes per warp; cap: slots a stage
// holds, at least the widest slice's).  The same arithmetic, rows and
// post() calls as slice_rows.  A stage whose copy has not landed after
// `spin_limit` polls sets *err to SFR_TIMEOUT and the warp goes on (its
// results are then meaningless and the caller reports the error).
template <int K, typename Acc, bool kExact, typename V, typename DV, typename I, int kStages,
          typename G, typename Pre, typename Post>
__device__ __forceinline__ void slice_rows_staged(int n, const int *sptr, const I *colp,
                                                  const V *valp, const DV *const *diagp, int s0,
                                                  int s1, int cap, char *smem, int *err,
                                                  const int (&act)[K], G g, Pre pre,
                                                  Post post) {
  using E = decltype(pre(0, 0));
  constexpr unsigned kSpinLimit = 1u << 24;
  const int lane = threadIdx.x & 31;
  const int warp = static_cast<int>(threadIdx.x >> 5);
  const int step = static_cast<int>(blockDim.x >> 5);
  char *base = smem + static_cast<size_t>(warp) * staged_warp_bytes<V, I, kStages>(cap);
  uint64_t *bar = reinterpret_cast<uint64_t *>(base);
  V *vs = reinterpret_cast<V *>(base + ((kStages * 8 + 15) / 16) * 16);
  I *cs = reinterpret_cast<I *>(vs + kStages * cap);
  const int first = s0 + warp;
  if (first >= s1) return;
  // lane 0: one slice into stage `stg`
  auto issue = [&](int s, int stg) {
    const int b = __ldg(sptr + s);
    const unsigned cnt = static_cast<unsigned>(__ldg(sptr + s + 1) - b);
    mbar_arrive_expect_tx(bar + stg, cnt * static_cast<unsigned>(sizeof(V) + sizeof(I)));
    if (cnt > 0) {
      bulk_copy_g2s(vs + stg * cap, valp + b, cnt * static_cast<unsigned>(sizeof(V)), bar + stg);
      bulk_copy_g2s(cs + stg * cap, colp + b, cnt * static_cast<unsigned>(sizeof(I)), bar + stg);
    }
  };
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < kStages; ++q) mbar_init(bar + q, 1);
    fence_proxy_async_smem();
#pragma unroll
    for (int q = 0; q < kStages; ++q)
      if (first + q * step < s1) issue(first + q * step, q);
  }
  __syncwarp();
  int i = 0;
  for (int s = first; s < s1; s += step, ++i) {
    const int stg = i % kStages;
    const unsigned parity = static_cast<unsigned>(i / kStages) & 1u;
    const int row = s * kWarp + lane;
    const int w = (__ldg(sptr + s + 1) - __ldg(sptr + s)) >> 5;
    E ex[K];
    Acc dv[K], gv[K];
    if (row < n) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (act[k]) {
          ex[k] = pre(k, row);
          dv[k] = static_cast<Acc>(ld_vec(diagp[k] + row));
          gv[k] = static_cast<Acc>(g(k, row));
        }
    }
    unsigned spins = 0;
    while (!mbar_try_wait(bar + stg, parity)) {
      if (++spins > kSpinLimit) {
        atomicCAS(err, 0, SFR_TIMEOUT);
        break;
      }
    }
    if (row < n) {
      const I *c = cs + stg * cap + lane;
      const V *v = vs + stg * cap + lane;
      Acc y[K];
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (act[k]) y[k] = kExact ? xmul(dv[k], gv[k]) : dv[k] * gv[k];
      for (int e0 = 0; e0 < w; e0 += 6) {
        int jj[6];
        Acc vv[6];
#pragma unroll
        for (int u = 0; u < 6; ++u)
          if (e0 + u < w) {
            jj[u] = smem_col(c, (e0 + u) * kWarp, row);
            vv[u] = static_cast<Acc>(v[(e0 + u) * kWarp]);
          }
#pragma unroll
        for (int u = 0; u < 6; ++u)
          if (e0 + u < w) {
#pragma unroll
            for (int k = 0; k < K; ++k)
              if (act[k]) {
                const Acc t = static_cast<Acc>(g(k, jj[u]));
                y[k] = kExact ? xadd(y[k], xmul(vv[u], t)) : fma(vv[u], t, y[k]);
              }
          }
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (act[k]) post(k, row, y[k], ex[k]);
    }
    __syncwarp();  // every lane is done with stage stg
    if (lane == 0 && s + kStages * step < s1) {
      fence_proxy_async_smem();
      issue(s + kStages * step, stg);
    }
  }
}

// Two operands of a row, the usual pre() result of slice_rows.
template <typename T>
struct RowPair {
  T a, b;
};

// Three per-row operands of a phase, loaded with the slice (slice_rows's pre)
template <typename T>
struct RowTriple {
  T a, b, c;
};

template <int K, bool kExact, typename V, typename G, typename I = int>
__device__ __forceinline__ void row_product(const int *sptr, const I *colp, const V *valp,
                                            const V *const *diagp, int s, int lane,
                                            const int (&act)[K], G g,
                                            typename std::conditional<kExact, double, float>::type (&y)[K]) {
  using T = typename std::conditional<kExact, double, float>::type;
  row_product_t<K, T, kExact, V, V, G, I>(sptr, colp, valp, diagp, s, lane, act, g, y);
}

// The same over SlotCols: the offset form when the pattern has it.
template <int K, bool kExact, typename V, typename G>
__device__ __forceinline__ void row_product(const int *sptr, const SlotCols &cols, const V *valp,
                                            const V *const *diagp, int s, int lane,
                                            const int (&act)[K], G g,
                                            typename std::conditional<kExact, double, float>::type (&y)[K]) {
  if (cols.off)
    row_product<K, kExact, V, G, int16_t>(sptr, cols.off, valp, diagp, s, lane, act, g, y);
  else
    row_product<K, kExact, V, G, int>(sptr, cols.col, valp, diagp, s, lane, act, g, y);
}
template <int K, typename Acc, bool kExact, typename V, typename DV, typename G>
__device__ __forceinline__ void row_product_t(const int *sptr, const SlotCols &cols,
                                              const V *valp, const DV *const *diagp, int s,
                                              int lane, const int (&act)[K], G g, Acc (&y)[K]) {
  if (cols.off)
    row_product_t<K, Acc, kExact, V, DV, G, int16_t>(sptr, cols.off, valp, diagp, s, lane, act,
                                                     g, y);
  else
    row_product_t<K, Acc, kExact, V, DV, G, int>(sptr, cols.col, valp, diagp, s, lane, act, g, y);
}

// Totals of NV values over `G` block partials, fixed order, all threads of
// the (last) block.  Result in sm[0..NV).
template <int NV>
__device__ __forceinline__ void block_totals(const double *part, int G, double *sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double s[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    s[v] = 0.0;
    for (int b = threadIdx.x; b < G; b += blockDim.x) s[v] += ld_vec(part + v * G + b);
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double w = warp_sum(s[v]);
    if (lane == 0) sm[32 + v * 32 + warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double w = lane < nw ? sm[32 + v * 32 + lane] : 0.0;
      w = warp_sum(w);
      if (lane == 0) sm[v] = w;
    }
  }
  __syncthreads();
}

// Block partials -> counter; true in the last block, with the totals in
// sm[0..NV) for every thread of that block.  The counter is reset there.
template <int NV>
__device__ __forceinline__ bool last_block(const double (&acc)[NV], double *part,
                                           unsigned *counter, double *sm) {
  __shared__ bool s_last;
  block_partials<NV>(acc, part, gridDim.x, sm + 32 + NV * 32);
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  block_totals<NV>(part, gridDim.x, sm);
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// Shared memory a last_block reduction of NV values needs.
#define SFR_SHARED_RED(NV) __shared__ double sm[32 + 2 * (NV) * 32]

// Block-contiguous slice range of this block.
__device__ __forceinline__ void block_slices(int nslices, int *first, int *last) {
  const long long G = gridDim.x;
  *first = static_cast<int>((static_cast<long long>(nslices) * blockIdx.x) / G);
  *last = static_cast<int>((static_cast<long long>(nslices) * (blockIdx.x + 1)) / G);
}

}  // namespace sfr
