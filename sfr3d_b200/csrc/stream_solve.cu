// Graph engine: a Krylov solve as one CUDA graph whose iteration loop is a
// device-controlled conditional WHILE node.
//
// Each phase of an iteration is its own full-occupancy kernel (one warp per
// SELL slice, a thread per row), so every row's loads are in flight at once;
// a phase's dot products end in the last block to finish, which sums the
// block partials in a fixed order (deterministic), updates the Krylov scalars
// in device memory and, from the last phase, sets the WHILE condition to 0
// once every right-hand side has stopped.  The host launches the graph and
// reads the result once: no per-iteration round trip.
//
// Loads: vectors are read with plain L1-cached loads (a warp's rows share
// most of their gathers); the matrix streams with evict-first.
//
// The persistent engine (krylov.cu, mixed.cu) suits small systems where
// launch latency dominates; this engine suits large ones.  Both follow the
// same arithmetic: FP64 rows and updates bit-identical to the reference
// (Cg.c, Bicgstab.c, HccaBlas.c), or FP32 inner iterations with FP64
// reliable updates (the true residual and x in FP64; the update kernels are
// plain graph nodes that return at once unless a refinement is due).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "persist.cuh"

namespace sfr {

namespace {

constexpr int kCounters = 16;

// The iteration's SpMV phases (k_pcg_a, k_bicg_a1, k_bicg_a2) trade a
// warp's loads in flight against warps resident.  slice_rows issues every
// load of a slice that does not depend on a column before the first gather
// (two dependent round trips a slice); it pays for that in registers.
// Measured at 128^3 (momentum K = 3, Poisson K = 1):
//   K = 1: slice_rows, uncapped (the three-kernel PCG 125.0 ms against
//          130.5 ms with row_product);
//   K > 1, FP32 operator: slice_rows capped at 4 blocks of 256 an SM
//          (64 registers; BiCGSTAB 4.67 ms against 5.16 ms);
//   K > 1, FP64: row_product (5.40 ms; slice_rows needs 97 registers and
//          ran 6.52 ms uncapped, 5.91 ms capped at 3 blocks, 7.23 ms at 4).
template <int K, bool kMixed>
struct SpmvShape {
  static constexpr bool kSliceRows = K == 1 || kMixed;
  static constexpr int kMinBlocks = (K > 1 && kMixed) ? 4 : 0;  // 0: no cap
};

template <int K>
struct SArgs {  // passed by value: every pointer is fixed for the graph's life
  int n, nslices, npairs;
  const int *sptr;
  SlotCols cols;  // slot columns (16-bit offsets when the bandwidth allows)
  const double *val64;
  const float *val32;
  // the graph's own padded workspace (rows padded to a multiple of 4)
  double *diag64[K], *b[K], *x[K];
  double *dc[K];        // mixed: diagonal of the FP32 operator, ad + compensation
  const double *comp;   // mixed: -sum_row (fl32(a_ij) - a_ij)
  double *m[K], *r[K], *z[K], *q[K], *p0[K], *p1[K], *r0[K], *t[K];
  float *m32[K], *fr[K], *fz[K], *fq[K], *fp0[K], *fp1[K], *fxs[K], *fr0[K], *ft[K];
  double *part;
  unsigned *counter;
  cudaGraphConditionalHandle hwhile;
  int in_graph;  // 0: plain launch loop (profiling): no conditional handles
  // the right-hand sides share one diagonal: diag64, m, dc and m32 of every
  // k point at k = 0's arrays, which k_setup fills once
  int shared_diag;
  // SpMV phases of the iteration: a warp prefetches into L2 the slice it
  // reaches `pf` rounds later (0: off)
  int pf;
  // BiCGSTAB's SpMV phases with the slices staged in shared memory by bulk
  // copies (kernels instantiated with kStages > 0): slots a stage holds, and
  // the word a stage wait that gave up sets
  int stage_cap;
  int *stage_err;
};


// Per-call scalars, copied into the state before each launch.
struct SCall {
  double tol, delta;
  unsigned maxit;
  int newx;
};

template <int K>
struct SState {
  SCall call;
  double d[K], alpha[K], beta[K], omega[K], rr0[K], conv[K], bnorm[K], rmax[K];
  int active[K], iters[K], status[K], refine[K], upd[K];
  int any, any_upd;
  unsigned j;
  SolveOut out[K];
};

// Vector phases run over row pairs (r, r+1) with 16-byte (FP64) / 8-byte
// (FP32) loads; every workspace vector is padded, so the pair is in bounds.
#define SFR_FOR_PAIRS(i)                                                        \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.npairs;             \
       i += gridDim.x * blockDim.x)

__device__ __forceinline__ double2 ld2(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ double2 ld2ro(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ float2 ld2ro(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(double *p, double2 v) { *reinterpret_cast<double2 *>(p) = v; }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }


template <int K>
__device__ __forceinline__ void load_active(const SState<K> *st, int (&act)[K]) {
#pragma unroll
  for (int k = 0; k < K; ++k) act[k] = st->active[k];
}

// ============================= PCG =======================================

// setup: m (and FP32 d/m), x0, (b, M^-1 b), (b, b)
template <int K, bool kMixed>
__global__ void __launch_bounds__(256) k_setup(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(2 * K);
  const int n = a.n;
  const int newx = st->call.newx;
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  SFR_FOR_PAIRS(i) {
    const int r = 2 * i;
    const bool two = r + 1 < n;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double2 dk = ld2ro(a.diag64[k] + r);
      const double2 mk = make_double2(1.0 / dk.x, 1.0 / dk.y);
      if (k == 0 || !a.shared_diag) {  // shared: k = 0's arrays serve every k
        if (kMixed) {
          const double2 ck = ld2ro(a.comp + r);
          st2(a.dc[k] + r, make_double2(dk.x + ck.x, dk.y + ck.y));
          st2(a.m32[k] + r, make_float2(__double2float_rn(mk.x), __double2float_rn(mk.y)));
        } else {
          st2(a.m[k] + r, mk);
        }
      }
      if (newx) st2(a.x[k] + r, make_double2(0.0, 0.0));
      const double2 bk = ld2ro(a.b[k] + r);
      acc[2 * k] += bk.x * xmul(bk.x, mk.x);
      acc[2 * k + 1] += bk.x * bk.x;
      if (two) {
        acc[2 * k] += bk.y * xmul(bk.y, mk.y);
        acc[2 * k + 1] += bk.y * bk.y;
      }
    }
  }
  if (!last_block<2 * K>(acc, a.part, a.counter + 0, sm)) return;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      st->conv[k] = st->call.tol * sqrt(fabs(sm[2 * k]));
      st->bnorm[k] = sqrt(sm[2 * k + 1]);
      st->active[k] = 1;
      st->iters[k] = 0;
      st->status[k] = SFR_OK;
      st->refine[k] = 0;
      st->upd[k] = 0;
      st->beta[k] = 0.0;
    }
    st->j = 0;
    st->any = 1;
    st->any_upd = 0;
  }
}

// PCG start: r = b - A x, z = M r, p = z, d = (r, z)  (FP64: Cg.c:84-102)
// mixed: the same in FP64 for the true residual, then r, z, p in FP32.
template <int K, bool kMixed, typename I>
__global__ void __launch_bounds__(256) k_pcg_start(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(2 * K);
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int all[K];
#pragma unroll
  for (int k = 0; k < K; ++k) all[k] = 1;
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  SFR_FOR_OWN_ROWS(s0, s1) {
    double y[K];
    row_product<K, true, double>(a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s_, lane, all,
                                 [&](int k, int c) { return ld_ro(a.x[k] + c); }, y);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double rk = xsub(ld_ro(a.b[k] + row_), y[k]);
      if (kMixed) {
        const float rs = __double2float_rn(rk);
        const float zs = ld_ro(a.m32[k] + row_) * rs;
        st_vec(a.fr[k] + row_, rs);
        st_vec(a.fz[k] + row_, zs);
        st_vec(a.fp0[k] + row_, zs);
        st_vec(a.fxs[k] + row_, 0.0f);
        acc[2 * k] += rk * (rk / ld_ro(a.diag64[k] + row_));
        acc[2 * k + 1] += static_cast<double>(rs) * static_cast<double>(zs);
      } else {
        const double zk = xmul(rk, ld_ro(a.m[k] + row_));
        st_vec(a.r[k] + row_, rk);
        st_vec(a.z[k] + row_, zk);
        st_vec(a.p0[k] + row_, zk);
        acc[2 * k + 1] += rk * zk;
      }
    }
  }
  if (!last_block<2 * K>(acc, a.part, a.counter + 1, sm)) return;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      st->d[k] = sm[2 * k + 1];
      st->rmax[k] = sqrt(fabs(sm[2 * k]));
    }
  }
}

// phase A: q = A p, (q, p)  (Cg.c:105-109)
template <int K, bool kMixed, typename I>
__global__ void __launch_bounds__(256, (SpmvShape<K, kMixed>::kMinBlocks)) k_pcg_a(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(K);
  if (!st->any) return;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int act[K];
  load_active<K>(st, act);
  const unsigned j = st->j;
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  if (!kMixed && !SpmvShape<K, kMixed>::kSliceRows) {
    SFR_FOR_OWN_ROWS(s0, s1) {
      prefetch_slice_ahead(a.pf, a.sptr, cols_of<I>(a.cols), a.val64, s_, s1);
      double y[K];
      row_product<K, true, double>(a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s_, lane, act,
                                   [&](int k, int c) { return ld_ro(a.p0[k] + c); }, y);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        st_vec(a.q[k] + row_, y[k]);
        acc[k] += y[k] * ld_ro(a.p0[k] + row_);
      }
    }
  } else if (!kMixed) {
    slice_rows<K, double, true, double, double, I>(
        n, a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s0, s1, a.pf, act,
        [&](int k, int c) { return ld_ro(a.p0[k] + c); },
        [&](int k, int row) { return ld_ro(a.p0[k] + row); },
        [&](int k, int row, double y, double pk) {
          st_vec(a.q[k] + row, y);
          acc[k] += y * pk;
        });
  } else {
    slice_rows<K, double, false, float, double, I>(
        n, a.sptr, cols_of<I>(a.cols), a.val32, a.dc, s0, s1, a.pf, act,
        [&](int k, int c) { return ld_ro(a.fp0[k] + c); },
        [&](int k, int row) { return ld_ro(a.fp0[k] + row); },
        [&](int k, int row, double y, float pk) {
          const float yf = __double2float_rn(y);
          st_vec(a.fq[k] + row, yf);
          acc[k] += static_cast<double>(yf) * static_cast<double>(pk);
        });
  }
  if (!last_block<K>(acc, a.part, a.counter + 2, sm)) return;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      const double al = st->d[k] / sm[k];
      st->alpha[k] = al;
      if (!isfinite(al)) {
        st->active[k] = 0;
        st->status[k] = SFR_BREAKDOWN;
        st->iters[k] = j + 1;
      }
    }
  }
}

// phase B: x (or xs) += alpha p ; r -= alpha q ; z = M r ; (r, z) ; test
template <int K, bool kMixed>
__global__ void __launch_bounds__(256) k_pcg_b(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(K);
  if (!st->any) return;
  const int n = a.n;
  int act[K];
  load_active<K>(st, act);
  const unsigned j = st->j;
  double acc[K], al[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    acc[k] = 0.0;
    al[k] = st->alpha[k];
  }
  SFR_FOR_PAIRS(i) {
    const int r = 2 * i;
    const bool two = r + 1 < n;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      if (!kMixed) {
        const double2 p = ld2ro(a.p0[k] + r), q = ld2ro(a.q[k] + r), m = ld2ro(a.m[k] + r);
        double2 xv = ld2(a.x[k] + r), rv = ld2(a.r[k] + r), zv;
        xv.x = xadd(xv.x, xmul(al[k], p.x));
        xv.y = xadd(xv.y, xmul(al[k], p.y));
        rv.x = xsub(rv.x, xmul(al[k], q.x));
        rv.y = xsub(rv.y, xmul(al[k], q.y));
        zv.x = xmul(rv.x, m.x);
        zv.y = xmul(rv.y, m.y);
        st2(a.x[k] + r, xv);
        st2(a.r[k] + r, rv);
        st2(a.z[k] + r, zv);
        acc[k] += rv.x * zv.x;
        if (two) acc[k] += rv.y * zv.y;
      } else {
        const float af = static_cast<float>(al[k]);
        const float2 p = ld2ro(a.fp0[k] + r), q = ld2ro(a.fq[k] + r), m = ld2ro(a.m32[k] + r);
        float2 xs = ld2(a.fxs[k] + r), rv = ld2(a.fr[k] + r), zv;
        xs.x = fmaf(af, p.x, xs.x);
        xs.y = fmaf(af, p.y, xs.y);
        rv.x = fmaf(-af, q.x, rv.x);
        rv.y = fmaf(-af, q.y, rv.y);
        zv.x = m.x * rv.x;
        zv.y = m.y * rv.y;
        st2(a.fxs[k] + r, xs);
        st2(a.fr[k] + r, rv);
        st2(a.fz[k] + r, zv);
        acc[k] += static_cast<double>(rv.x) * static_cast<double>(zv.x);
        if (two) acc[k] += static_cast<double>(rv.y) * static_cast<double>(zv.y);
      }
    }
  }
  if (!last_block<K>(acc, a.part, a.counter + 3, sm)) return;
  if (threadIdx.x == 0) {
    int any = 0, any_upd = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      st->upd[k] = 0;
      if (!act[k]) continue;
      const double di = sm[k];
      if (!kMixed) {
        st->beta[k] = di / st->d[k];
        st->d[k] = di;
        if (sqrt(fabs(di)) < st->conv[k]) {
          st->active[k] = 0;
          st->iters[k] = j + 1;
        } else if (!isfinite(st->beta[k])) {
          st->active[k] = 0;
          st->status[k] = SFR_BREAKDOWN;
          st->iters[k] = j + 1;
        }
      } else {
        const double est = sqrt(fabs(di));
        if (!isfinite(di)) {
          st->active[k] = 0;
          st->status[k] = SFR_BREAKDOWN;
          st->iters[k] = j + 1;
        } else if (est < st->call.delta * st->rmax[k] || est < st->conv[k]) {
          st->upd[k] = 1;
          any_upd = 1;
        } else {
          st->beta[k] = di / st->d[k];
          st->d[k] = di;
        }
      }
      if (st->active[k] && !st->upd[k] && j + 1 >= st->call.maxit) {
        st->active[k] = 0;
        st->status[k] = SFR_MAXIT;
        st->iters[k] = j + 2;
      }
      any |= st->active[k];
    }
    st->j = j + 1;
    st->any = any;
    st->any_upd = any_upd;
    if (!any && a.in_graph) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// phase C: p = z + beta p  (Cg.c:139-141), in place
template <int K, bool kMixed>
__global__ void __launch_bounds__(256) k_pcg_c(const SArgs<K> a, SState<K> *st) {
  if (!st->any) return;
  int act[K];
  load_active<K>(st, act);
  double bv[K];
#pragma unroll
  for (int k = 0; k < K; ++k) bv[k] = st->beta[k];
  SFR_FOR_PAIRS(i) {
    const int r = 2 * i;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      if (!kMixed) {
        const double2 zv = ld2ro(a.z[k] + r);
        double2 p = ld2(a.p0[k] + r);
        p.x = xadd(zv.x, xmul(bv[k], p.x));
        p.y = xadd(zv.y, xmul(bv[k], p.y));
        st2(a.p0[k] + r, p);
      } else {
        const float bf = static_cast<float>(bv[k]);
        const float2 zv = ld2ro(a.fz[k] + r);
        float2 p = ld2(a.fp0[k] + r);
        p.x = fmaf(bf, p.x, zv.x);
        p.y = fmaf(bf, p.y, zv.y);
        st2(a.fp0[k] + r, p);
      }
    }
  }
}

// Partial sums of a co-resident grid, reduced once and broadcast: every block
// stores its total in part[b], then arrives at one counter; the last block
// to arrive sums the G totals in a fixed order and publishes the sum in one
// word whose two lowest bits carry the epoch's tag (epoch & 3, at most 3
// units in the last place), after resetting the counter; every other block
// polls that word (acquire) until it carries the tag.  So the G partials are read once
// (by the last block) instead of by every block, and the waiters' one poll
// brings the value.  The word is rewritten every epoch; a waiter for epoch e
// finds there epoch e-1's sum (another tag) until e's arrives.  It starts
// each solve at zero and epochs start at 1.  Only the partial sums cross: no
// other global data is ordered by it.  A wait gives up after spin_limit polls
// and records SFR_TIMEOUT in *err.
struct TagExchange {
  unsigned long long *word;  // the broadcast word, zero at the start of a solve
  unsigned *count;           // arrivals, zero between exchanges
  int *err;
  unsigned spin_limit;
};

__device__ __forceinline__ bool tag_exchange(const TagExchange &x, unsigned epoch, double v,
                                             double *part, double *total, double *sm) {
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int G = gridDim.x;
  const double wsum = warp_sum(v);
  if (lane == 0) sm[warp] = wsum;
  __syncthreads();
  const unsigned tag = epoch & 3u;
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> word(*x.word);
  cuda::atomic_ref<int, cuda::thread_scope_device> err(*x.err);
  if (warp == 0) {
    const double bt = warp_sum(lane < nw ? sm[lane] : 0.0);
    if (lane == 0) {
      st_vec(part + blockIdx.x, bt);
      // release: the partial above is visible before the arrival counts
      s_last = cuda::atomic_ref<unsigned, cuda::thread_scope_device>(*x.count)
                   .fetch_add(1u, cuda::memory_order_acq_rel) == static_cast<unsigned>(G) - 1u;
    }
  }
  __syncthreads();
  bool ok = true;
  if (s_last) {
    // every thread of the last block loads its share of the G partials at
    // once (one L2 round trip), then the block sums them in a fixed order:
    // thread t's partials t, t + blockDim.x, ... in turn, the warps' shuffle
    // trees, the warps in order
    cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
    constexpr int kAhead = 5;
    double pv[kAhead];
#pragma unroll
    for (int q = 0; q < kAhead; ++q) {
      const int b = static_cast<int>(threadIdx.x) + q * static_cast<int>(blockDim.x);
      pv[q] = b < G ? __ldcg(part + b) : 0.0;
    }
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < kAhead; ++q) t += pv[q];
    for (int b = static_cast<int>(threadIdx.x) + kAhead * static_cast<int>(blockDim.x); b < G;
         b += blockDim.x)
      t += __ldcg(part + b);
    t = warp_sum(t);
    if (lane == 0) sm[warp] = t;
    __syncthreads();
    if (warp == 0) {
      t = warp_sum(lane < nw ? sm[lane] : 0.0);
      if (lane == 0) {
        *x.count = 0u;
        const unsigned long long u =
            (static_cast<unsigned long long>(__double_as_longlong(t)) & ~3ull) | tag;
        word.store(u, cuda::memory_order_release);
        sm[32] = __longlong_as_double(static_cast<long long>(u));
      }
    }
  } else if (threadIdx.x == 0) {
    for (unsigned spins = 0;; ++spins) {
      // acquire: the counter's reset before the publication is visible to
      // this block's next arrival
      const unsigned long long u = word.load(cuda::memory_order_acquire);
      if ((u & 3ull) == tag) {
        sm[32] = __longlong_as_double(static_cast<long long>(u));
        break;
      }
      if (err.load(cuda::memory_order_relaxed) != 0) {
        ok = false;
        break;
      }
      if (spins > x.spin_limit) {
        int expected = 0;
        err.compare_exchange_strong(expected, SFR_TIMEOUT, cuda::memory_order_relaxed);
        ok = false;
        break;
      }
    }
    if (!ok) sm[33] = 1.0;
  }
  if (threadIdx.x == 0 && ok) sm[33] = 0.0;
  __syncthreads();
  *total = sm[32];
  ok = sm[33] == 0.0;
  __syncthreads();
  return ok;
}

// One whole FP64 PCG iteration (one right-hand side) in one cooperative
// launch: the three phases above with two grid barriers between them instead
// of kernel boundaries.  A block keeps q = A p of its own rows in shared
// memory from phase A to phase B, and then z = M r in the same words from
// phase B to phase C, so neither q nor z crosses HBM; the block's p is still
// in cache when phase C rewrites it.  Each barrier's dot product is reduced
// by every block over all block partials in the same fixed order, so every
// block holds the same alpha, beta and stop decision.  Every row is computed
// with the same expressions as in k_pcg_a/b/c (bit-identical rows).
// The barriers are bounded: a wait that gives up records SFR_TIMEOUT, every
// block leaves, and the solve stops with that status.
// kTagged: the barriers are tag_exchange (mode 3: the last block reduces and
// broadcasts) instead of grid_sync with every block reading the partials.
// Iteration j from d = (r, z); returns true with d = the new (r, z) when the
// solve goes on, false when it stopped (converged, breakdown, iteration cap
// or a wait that gave up), with the state recorded by block 0.

// Stops the fused solve with `status` after `iters` iterations (block 0
// records it).
__device__ __forceinline__ void fused_stop(const SArgs<1> &a, SState<1> *st, int status,
                                           unsigned iters) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->active[0] = 0;
    st->status[0] = status;
    st->iters[0] = static_cast<int>(iters);
    st->any = 0;
    if (a.in_graph) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

template <typename I, bool kTagged>
__device__ __forceinline__ bool pcg_fused_body(const SArgs<1> &a, SState<1> *st,
                                               const GridSync &gs, const TagExchange &tx,
                                               const unsigned j, double &d_io) {
  __shared__ double sm[34 * 2];
  extern __shared__ double qz[];  // this block's rows: q, then z
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int row0 = s0 * kWarp;
  const int all[1] = {1};
  const double d = d_io;
  const int G = gridDim.x;
  auto fail = [&](int status, unsigned iters) { fused_stop(a, st, status, iters); };
  // phase A: q = A p, (p, q); each slice's column-independent loads go out
  // with its columns (slice_rows: 114.6 -> 106.9 ms a 128^3 solve in mode 3)
  double acc[1] = {0.0};
  slice_rows<1, double, true, double, double, I>(
      n, a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s0, s1, 0, all,
      [&](int, int c) { return ld_ro(a.p0[0] + c); },
      [&](int, int row) { return ld_ro(a.p0[0] + row); },
      [&](int, int row, double y, double pk) {
        qz[row - row0] = y;
        acc[0] += y * pk;
      });
  double tot[1];
  if (kTagged) {
    if (!tag_exchange(tx, 2 * j + 1, acc[0], a.part, &tot[0], sm)) {
      fail(SFR_TIMEOUT, j + 1);
      return false;
    }
  } else {
    block_partials<1>(acc, a.part, G, sm);
    if (!grid_sync(gs)) {
      fail(SFR_TIMEOUT, j + 1);
      return false;
    }
    grid_totals<1>(a.part, G, G, tot, sm);
  }
  const double alpha = d / tot[0];
  if (!isfinite(alpha)) {
    fail(SFR_BREAKDOWN, j + 1);
    return false;
  }
  // phase B: x += alpha p, r -= alpha q, z = M r, (r, z)
  acc[0] = 0.0;
  SFR_FOR_OWN_ROWS(s0, s1) {
    const double p = ld_ro(a.p0[0] + row_);
    const double xv = xadd(ld_vec(a.x[0] + row_), xmul(alpha, p));
    const double rv = xsub(ld_vec(a.r[0] + row_), xmul(alpha, qz[row_ - row0]));
    const double zv = xmul(rv, ld_ro(a.m[0] + row_));
    st_vec(a.x[0] + row_, xv);
    st_vec(a.r[0] + row_, rv);
    qz[row_ - row0] = zv;
    acc[0] += rv * zv;
  }
  if (kTagged) {
    if (!tag_exchange(tx, 2 * j + 2, acc[0], a.part + G, &tot[0], sm)) {
      fail(SFR_TIMEOUT, j + 1);
      return false;
    }
  } else {
    block_partials<1>(acc, a.part + G, G, sm);
    if (!grid_sync(gs)) {
      fail(SFR_TIMEOUT, j + 1);
      return false;
    }
    grid_totals<1>(a.part + G, G, G, tot, sm);
  }
  const double di = tot[0];
  const double beta = di / d;
  bool stop = false;
  int status = SFR_OK;
  unsigned iters = 0;
  if (sqrt(fabs(di)) < st->conv[0]) {
    stop = true;
    iters = j + 1;
  } else if (!isfinite(beta)) {
    stop = true;
    status = SFR_BREAKDOWN;
    iters = j + 1;
  } else if (j + 1 >= st->call.maxit) {
    stop = true;
    status = SFR_MAXIT;
    iters = j + 2;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->alpha[0] = alpha;
    st->beta[0] = beta;
    st->d[0] = di;
    st->j = j + 1;
    if (stop) {
      st->active[0] = 0;
      st->status[0] = status;
      st->iters[0] = static_cast<int>(iters);
      st->any = 0;
      if (a.in_graph) cudaGraphSetConditional(a.hwhile, 0u);
    }
  }
  if (stop) return false;
  // phase C: p = z + beta p
  SFR_FOR_OWN_ROWS(s0, s1) {
    const double p = ld_ro(a.p0[0] + row_);
    st_vec(a.p0[0] + row_, xadd(qz[row_ - row0], xmul(beta, p)));
  }
  d_io = di;
  return true;
}

// The fused iteration as launched: mode 1 leaves the register count to the
// compiler (48), mode 2 holds it to 40 so that six blocks fit an SM, mode 3
// is mode 1 with the tagged exchanges.
template <typename I, int kMode>
__global__ void __launch_bounds__(256) k_pcg_fused(const SArgs<1> a, SState<1> *st, GridSync gs,
                                                   TagExchange tx, unsigned *) {
  if (!st->any) return;
  double d = st->d[0];
  (void)pcg_fused_body<I, kMode == 3>(a, st, gs, tx, st->j, d);
}
template <typename I>
__global__ void __launch_bounds__(256, 6) k_pcg_fused_r40(const SArgs<1> a, SState<1> *st,
                                                          GridSync gs, TagExchange tx, unsigned *) {
  if (!st->any) return;
  double d = st->d[0];
  (void)pcg_fused_body<I, false>(a, st, gs, tx, st->j, d);
}

// Mode 4: the whole solve in one cooperative launch, mode 3's iteration in a
// loop.  The kernel boundary that published p between iterations becomes a
// wait on the blocks whose p the next SpMV phase gathers (neighbour_wait;
// the two exchanges inside an iteration keep every block from rewriting p
// while another still reads it).  A block finds those blocks once, from the
// columns of its slices.  Held to four blocks an SM (64 registers): 91.9 ms
// a 128^3 solve, against 97.2 ms with the compiler's own choice at the same
// register count, 103.2 ms at three blocks and 119.4 ms at five.
template <typename I>
__global__ void __launch_bounds__(256, 4) k_pcg_fused_loop(const SArgs<1> a, SState<1> *st,
                                                           GridSync gs, TagExchange tx,
                                                           unsigned *ticks) {
  __shared__ int range[2];
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    int cmin = s0 * kWarp, cmax = s1 * kWarp - 1;
    const I *cols = cols_of<I>(a.cols);
    for (int s = s0 + static_cast<int>(threadIdx.x >> 5); s < s1; s += nw) {
      const int base = __ldg(a.sptr + s), w = (__ldg(a.sptr + s + 1) - base) >> 5;
      const int row = s * kWarp + lane;
      for (int k = 0; k < w; ++k) {
        const int c = slot_col(cols + base + lane, k * kWarp, row);
        cmin = min(cmin, c);
        cmax = max(cmax, c);
      }
    }
    if (threadIdx.x == 0) {
      range[0] = cmin;
      range[1] = cmax;
    }
    __syncthreads();
    atomicMin(range, cmin);
    atomicMax(range + 1, cmax);
    __syncthreads();
    const int lo = min(owner_block(range[0], a.nslices), static_cast<int>(blockIdx.x));
    const int hi = max(owner_block(range[1], a.nslices), static_cast<int>(blockIdx.x));
    __syncthreads();
    if (threadIdx.x == 0) {
      range[0] = lo;
      range[1] = hi;
    }
    __syncthreads();
  }
  if (!st->any) return;
  unsigned j = st->j;
  double d = st->d[0];
  const bool local = range[1] - range[0] < static_cast<int>(blockDim.x);
  while (pcg_fused_body<I, true>(a, st, gs, tx, j, d)) {
    const bool ok = local ? neighbour_wait(ticks, tx.err, tx.spin_limit, j + 1, range[0], range[1])
                          : grid_sync(gs);
    if (!ok) {
      fused_stop(a, st, SFR_TIMEOUT, j + 1);
      return;
    }
    ++j;
  }
}

// The fused kernel of a mode.
template <typename I>
const void *fused_kernel(int mode) {
  return mode == 2   ? (const void *)k_pcg_fused_r40<I>
         : mode == 3 ? (const void *)k_pcg_fused<I, 3>
         : mode == 4 ? (const void *)k_pcg_fused_loop<I>
                     : (const void *)k_pcg_fused<I, 1>;
}

// Self-test of the bounded waits: the grid meets once at a grid_sync (kind
// 0) or a tag_exchange (kind 1), except its last `absent` blocks, which
// leave before it, so the others' wait on them runs out and records
// SFR_TIMEOUT.
__global__ void k_wait_selftest(int kind, int absent, GridSync gs, TagExchange tx, double *part) {
  __shared__ double sm[34];
  if (static_cast<int>(blockIdx.x) >= static_cast<int>(gridDim.x) - absent) return;
  if (kind == 0) {
    (void)grid_sync(gs);
  } else {
    double tot = 0.0;
    (void)tag_exchange(tx, 1u, 1.0, part, &tot, sm);
  }
}

// reliable update, part 1: x += xs (FP64) for the flagged right-hand sides
template <int K>
__global__ void __launch_bounds__(256) k_fold(const SArgs<K> a, SState<K> *st, int all) {
  if (!all && !st->any_upd) return;
  int sel[K];
#pragma unroll
  for (int k = 0; k < K; ++k) sel[k] = all ? 1 : st->upd[k];
  SFR_FOR_PAIRS(i) {
    const int r = 2 * i;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!sel[k]) continue;
      double2 xv = ld2(a.x[k] + r);
      const float2 xs = ld2(a.fxs[k] + r);
      xv.x += static_cast<double>(xs.x);
      xv.y += static_cast<double>(xs.y);
      st2(a.x[k] + r, xv);
      if (all) st2(a.fxs[k] + r, make_float2(0.f, 0.f));
    }
  }
}

// reliable update, part 2 (PCG): r_true = b - A x in FP64, r = fl32(r_true),
// z = M r, xs = 0; decide on the true residual.
template <int K, typename I>
__global__ void __launch_bounds__(256) k_pcg_refresh(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(2 * K);
  if (!st->any_upd) return;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int sel[K];
#pragma unroll
  for (int k = 0; k < K; ++k) sel[k] = st->upd[k];
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  SFR_FOR_OWN_ROWS(s0, s1) {
    double y[K];
    row_product<K, true, double>(a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s_, lane, sel,
                                 [&](int k, int c) { return ld_ro(a.x[k] + c); }, y);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!sel[k]) continue;
      const double rt = ld_ro(a.b[k] + row_) - y[k];
      const float rs = __double2float_rn(rt);
      const float zs = ld_ro(a.m32[k] + row_) * rs;
      st_vec(a.fr[k] + row_, rs);
      st_vec(a.fz[k] + row_, zs);
      st_vec(a.fxs[k] + row_, 0.0f);
      acc[2 * k] += rt * (rt / ld_ro(a.diag64[k] + row_));
      acc[2 * k + 1] += static_cast<double>(rs) * static_cast<double>(zs);
    }
  }
  if (!last_block<2 * K>(acc, a.part, a.counter + 4, sm)) return;
  if (threadIdx.x == 0) {
    const unsigned j = st->j;  // already advanced by phase B
    int any = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (sel[k]) {
        st->refine[k] += 1;
        st->upd[k] = 0;
        const double tr = sqrt(fabs(sm[2 * k]));
        if (tr < st->conv[k]) {
          st->active[k] = 0;
          st->iters[k] = j;
        } else {
          st->beta[k] = sm[2 * k + 1] / st->d[k];
          st->d[k] = sm[2 * k + 1];
          st->rmax[k] = tr;
          if (j >= st->call.maxit) {
            st->active[k] = 0;
            st->status[k] = SFR_MAXIT;
            st->iters[k] = j + 1;
          }
        }
      }
      any |= st->active[k];
    }
    st->any = any;
    st->any_upd = 0;
    if (!any && a.in_graph) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// post-processing: xKx, ||x||, ||b - Ax||_M, ||b - Ax|| (Cg.c:155-176)
template <int K, typename I>
__global__ void __launch_bounds__(256) k_post(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(4 * K);
  const int n = a.n;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int all[K];
#pragma unroll
  for (int k = 0; k < K; ++k) all[k] = 1;
  double acc[4 * K];
#pragma unroll
  for (int v = 0; v < 4 * K; ++v) acc[v] = 0.0;
  // the row's x, b and diagonal load with the slice
  slice_rows<K, double, true, double, double, I>(
      n, a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s0, s1, 0, all,
      [&](int k, int c) { return ld_ro(a.x[k] + c); },
      [&](int k, int row) {
        return RowTriple<double>{ld_ro(a.x[k] + row), ld_ro(a.b[k] + row),
                                 ld_ro(a.diag64[k] + row)};
      },
      [&](int k, int row, double y, RowTriple<double> e) {
        const double rk = xsub(e.b, y);
        acc[4 * k + 0] += e.a * y;
        acc[4 * k + 1] += e.a * e.a;
        acc[4 * k + 2] += rk * xmul(rk, 1.0 / e.c);
        acc[4 * k + 3] += rk * rk;
      });
  if (!last_block<4 * K>(acc, a.part, a.counter + 7, sm)) return;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      SolveOut o;
      o.iters = st->iters[k];
      o.status = st->status[k];
      o.xKx = sm[4 * k];
      o.norm_x = sqrt(sm[4 * k + 1]);
      o.norm_r_m = sqrt(fabs(sm[4 * k + 2]));
      o.norm_r = sqrt(sm[4 * k + 3]);
      o.conv = st->conv[k];
      o.bnorm = st->bnorm[k];
      o.refinements = st->refine[k];
      o.inner_iters = st->iters[k];
      o.team_ms = 0.0;
      if (a.stage_err && *a.stage_err != 0) o.status = SFR_TIMEOUT;  // a stage wait gave up
      st->out[k] = o;
    }
  }
}

// =========================== BiCGSTAB ====================================
// FP64: Bicgstab.c:50-245.  Vectors: r0 shadow, p (p0), z = M p or M s,
// v (q), t.  Mixed: the same in FP32 with xs and reliable updates.

template <int K, bool kMixed, typename I>
__global__ void __launch_bounds__(256) k_bicg_start(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(2 * K);
  const int n = a.n;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int all[K];
#pragma unroll
  for (int k = 0; k < K; ++k) all[k] = 1;
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  // the row's b and M (FP32 M held exactly as a double) load with the slice
  slice_rows<K, double, true, double, double, I>(
      n, a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s0, s1, 0, all,
      [&](int k, int c) { return ld_ro(a.x[k] + c); },
      [&](int k, int row) {
        return RowPair<double>{ld_ro(a.b[k] + row),
                               kMixed ? static_cast<double>(ld_ro(a.m32[k] + row))
                                      : ld_ro(a.m[k] + row)};
      },
      [&](int k, int row, double y, RowPair<double> e) {
        const double rk = xsub(e.a, y);
        if (kMixed) {
          const float rs = __double2float_rn(rk);
          st_vec(a.fr0[k] + row, rs);
          st_vec(a.fp0[k] + row, rs);
          st_vec(a.fr[k] + row, rs);
          st_vec(a.fz[k] + row, static_cast<float>(e.b) * rs);
          st_vec(a.fxs[k] + row, 0.0f);
        } else {
          st_vec(a.r0[k] + row, rk);
          st_vec(a.p0[k] + row, rk);
          st_vec(a.r[k] + row, rk);
          st_vec(a.z[k] + row, xmul(rk, e.b));
        }
        acc[2 * k] += rk * rk;
      });
  if (!last_block<2 * K>(acc, a.part, a.counter + 1, sm)) return;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      st->rmax[k] = sqrt(sm[2 * k]);
      st->conv[k] = st->call.tol * st->bnorm[k];  // ||r|| < tol ||b|| (Bicgstab.c:72-80)
    }
  }
}

// A1: v = A z ; rr0 = (r, r0) ; alpha = rr0 / (v, r0)
template <int K, bool kMixed, typename I, int kStages = 0>
__global__ void __launch_bounds__(256, (SpmvShape<K, kMixed>::kMinBlocks)) k_bicg_a1(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(2 * K);
  if (!st->any) return;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int act[K];
  load_active<K>(st, act);
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  auto g64 = [&](int k, int c) { return ld_ro(a.z[k] + c); };
  auto pre64 = [&](int k, int row) {
    return RowPair<double>{ld_ro(a.r[k] + row), ld_ro(a.r0[k] + row)};
  };
  auto post64 = [&](int k, int row, double y, RowPair<double> e) {
    st_vec(a.q[k] + row, y);
    acc[2 * k] += e.a * e.b;
    acc[2 * k + 1] += y * e.b;
  };
  // FP32 accumulation: the momentum systems BiCGSTAB serves are diagonally
  // dominant, and FP64 accumulation of K right-hand sides costs two FP32 ->
  // FP64 conversions a slot and right-hand side (the SpMV phase then ran
  // slower than the FP64 one)
  auto g32 = [&](int k, int c) { return ld_ro(a.fz[k] + c); };
  auto pre32 = [&](int k, int row) {
    return RowPair<float>{ld_ro(a.fr[k] + row), ld_ro(a.fr0[k] + row)};
  };
  auto post32 = [&](int k, int row, float y, RowPair<float> e) {
    st_vec(a.fq[k] + row, y);
    const double r0k = e.b;
    acc[2 * k] += static_cast<double>(e.a) * r0k;
    acc[2 * k + 1] += static_cast<double>(y) * r0k;
  };
  if constexpr (kStages > 0) {
    extern __shared__ __align__(16) char stage_smem[];
    if constexpr (!kMixed)
      slice_rows_staged<K, double, true, double, double, I, kStages>(
          n, a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s0, s1, a.stage_cap, stage_smem,
          a.stage_err, act, g64, pre64, post64);
    else
      slice_rows_staged<K, float, false, float, double, I, kStages>(
          n, a.sptr, cols_of<I>(a.cols), a.val32, a.dc, s0, s1, a.stage_cap, stage_smem,
          a.stage_err, act, g32, pre32, post32);
  } else if constexpr (!kMixed && !SpmvShape<K, kMixed>::kSliceRows) {
    SFR_FOR_OWN_ROWS(s0, s1) {
      prefetch_slice_ahead(a.pf, a.sptr, cols_of<I>(a.cols), a.val64, s_, s1);
      double y[K];
      row_product<K, true, double>(a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s_, lane, act,
                                   g64, y);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        st_vec(a.q[k] + row_, y[k]);
        const double r0k = ld_ro(a.r0[k] + row_);
        acc[2 * k] += ld_ro(a.r[k] + row_) * r0k;
        acc[2 * k + 1] += y[k] * r0k;
      }
    }
  } else if constexpr (!kMixed) {
    slice_rows<K, double, true, double, double, I>(n, a.sptr, cols_of<I>(a.cols), a.val64,
                                                   a.diag64, s0, s1, a.pf, act, g64, pre64,
                                                   post64);
  } else {
    slice_rows<K, float, false, float, double, I>(n, a.sptr, cols_of<I>(a.cols), a.val32, a.dc,
                                                  s0, s1, a.pf, act, g32, pre32, post32);
  }
  if (!last_block<2 * K>(acc, a.part, a.counter + 2, sm)) return;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      st->rr0[k] = sm[2 * k];
      st->alpha[k] = sm[2 * k] / sm[2 * k + 1];
      if (!isfinite(st->alpha[k])) {
        st->active[k] = 0;
        st->status[k] = SFR_BREAKDOWN;
        st->iters[k] = st->j + 1;
      }
    }
  }
}

// B1: x += alpha z ; s = r -= alpha v ; z = M s ; (s, s) ; half-step test
template <int K, bool kMixed>
__global__ void __launch_bounds__(256) k_bicg_b1(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(K);
  if (!st->any) return;
  const int n = a.n;
  int act[K];
  load_active<K>(st, act);
  double acc[K], alv[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    acc[k] = 0.0;
    alv[k] = st->alpha[k];
  }
  SFR_FOR_PAIRS(i) {
    const int r = 2 * i;
    const bool two = r + 1 < n;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      if (!kMixed) {
        const double al = alv[k];
        const double2 zv = ld2(a.z[k] + r), q = ld2ro(a.q[k] + r), m = ld2ro(a.m[k] + r);
        double2 xv = ld2(a.x[k] + r), rv = ld2(a.r[k] + r);
        xv.x = xadd(xv.x, xmul(al, zv.x));
        xv.y = xadd(xv.y, xmul(al, zv.y));
        rv.x = xsub(rv.x, xmul(al, q.x));
        rv.y = xsub(rv.y, xmul(al, q.y));
        st2(a.x[k] + r, xv);
        st2(a.r[k] + r, rv);
        st2(a.z[k] + r, make_double2(xmul(rv.x, m.x), xmul(rv.y, m.y)));
        acc[k] += rv.x * rv.x;
        if (two) acc[k] += rv.y * rv.y;
      } else {
        const float af = static_cast<float>(alv[k]);
        const float2 zv = ld2(a.fz[k] + r), q = ld2ro(a.fq[k] + r), m = ld2ro(a.m32[k] + r);
        float2 xs = ld2(a.fxs[k] + r), rv = ld2(a.fr[k] + r);
        xs.x = fmaf(af, zv.x, xs.x);
        xs.y = fmaf(af, zv.y, xs.y);
        rv.x = fmaf(-af, q.x, rv.x);
        rv.y = fmaf(-af, q.y, rv.y);
        st2(a.fxs[k] + r, xs);
        st2(a.fr[k] + r, rv);
        st2(a.fz[k] + r, make_float2(m.x * rv.x, m.y * rv.y));
        acc[k] += static_cast<double>(rv.x) * static_cast<double>(rv.x);
        if (two) acc[k] += static_cast<double>(rv.y) * static_cast<double>(rv.y);
      }
    }
  }
  if (!last_block<K>(acc, a.part, a.counter + 3, sm)) return;
  if (threadIdx.x == 0) {
    int any = 0, any_upd = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      st->upd[k] = 0;
      if (!act[k]) continue;
      if (sqrt(sm[k]) < st->conv[k]) {
        if (kMixed) {
          st->upd[k] = 1;  // confirm on the FP64 true residual
          any_upd = 1;
        } else {
          st->active[k] = 0;
          st->iters[k] = st->j + 1;
        }
      }
      any |= st->active[k];
    }
    st->any = any;
    st->any_upd = any_upd;
    if (!any && a.in_graph) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// reliable update (BiCGSTAB): r_true = b - A x, r = fl32(r_true), z = M r,
// xs = 0; ||r_true||; (r, r0).  `stage` 1 = after the half step, 2 = after
// the full step (phase B2 already computed beta; it is recomputed with the
// new (r, r0)).
template <int K, typename I>
__global__ void __launch_bounds__(256) k_bicg_refresh(const SArgs<K> a, SState<K> *st,
                                                      int stage) {
  SFR_SHARED_RED(2 * K);
  if (!st->any_upd) return;
  const int n = a.n;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int sel[K];
#pragma unroll
  for (int k = 0; k < K; ++k) sel[k] = st->upd[k];
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  // the row's b, r0 and M (FP32 held exactly as doubles) load with the slice
  slice_rows<K, double, true, double, double, I>(
      n, a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s0, s1, 0, sel,
      [&](int k, int c) { return ld_ro(a.x[k] + c); },
      [&](int k, int row) {
        return RowTriple<double>{ld_ro(a.b[k] + row), static_cast<double>(ld_ro(a.fr0[k] + row)),
                                 static_cast<double>(ld_ro(a.m32[k] + row))};
      },
      [&](int k, int row, double y, RowTriple<double> e) {
        const double rt = e.a - y;
        const float rs = __double2float_rn(rt);
        st_vec(a.fr[k] + row, rs);
        st_vec(a.fz[k] + row, static_cast<float>(e.c) * rs);
        st_vec(a.fxs[k] + row, 0.0f);
        acc[2 * k] += rt * rt;
        acc[2 * k + 1] += static_cast<double>(rs) * e.b;
      });
  if (!last_block<2 * K>(acc, a.part, a.counter + 4, sm)) return;
  if (threadIdx.x == 0) {
    const unsigned j = st->j;
    int any = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (sel[k]) {
        st->refine[k] += 1;
        st->upd[k] = 0;
        const double tr = sqrt(sm[2 * k]);
        if (tr < st->conv[k]) {
          st->active[k] = 0;
          st->iters[k] = stage == 1 ? j + 1 : j;
        } else {
          st->rmax[k] = tr;
          if (stage == 2) {
            st->beta[k] = (sm[2 * k + 1] / st->rr0[k]) * (st->alpha[k] / st->omega[k]);
            if (j >= st->call.maxit) {
              st->active[k] = 0;
              st->status[k] = SFR_MAXIT;
              st->iters[k] = j + 1;
            }
          }
        }
      }
      any |= st->active[k];
    }
    st->any = any;
    st->any_upd = 0;
    if (!any && a.in_graph) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// A2: t = A z ; w = (t, s) / (t, t)
template <int K, bool kMixed, typename I, int kStages = 0>
__global__ void __launch_bounds__(256, (SpmvShape<K, kMixed>::kMinBlocks)) k_bicg_a2(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(2 * K);
  if (!st->any) return;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  int act[K];
  load_active<K>(st, act);
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  auto g64 = [&](int k, int c) { return ld_ro(a.z[k] + c); };
  auto pre64 = [&](int k, int row) { return ld_ro(a.r[k] + row); };
  auto post64 = [&](int k, int row, double y, double rk) {
    st_vec(a.t[k] + row, y);
    acc[2 * k] += y * rk;
    acc[2 * k + 1] += y * y;
  };
  // FP32 accumulation, as in phase A1
  auto g32 = [&](int k, int c) { return ld_ro(a.fz[k] + c); };
  auto pre32 = [&](int k, int row) { return ld_ro(a.fr[k] + row); };
  auto post32 = [&](int k, int row, float y, float rk) {
    st_vec(a.ft[k] + row, y);
    acc[2 * k] += static_cast<double>(y) * static_cast<double>(rk);
    acc[2 * k + 1] += static_cast<double>(y) * static_cast<double>(y);
  };
  if constexpr (kStages > 0) {
    extern __shared__ __align__(16) char stage_smem[];
    if constexpr (!kMixed)
      slice_rows_staged<K, double, true, double, double, I, kStages>(
          n, a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s0, s1, a.stage_cap, stage_smem,
          a.stage_err, act, g64, pre64, post64);
    else
      slice_rows_staged<K, float, false, float, double, I, kStages>(
          n, a.sptr, cols_of<I>(a.cols), a.val32, a.dc, s0, s1, a.stage_cap, stage_smem,
          a.stage_err, act, g32, pre32, post32);
  } else if constexpr (!kMixed && !SpmvShape<K, kMixed>::kSliceRows) {
    SFR_FOR_OWN_ROWS(s0, s1) {
      prefetch_slice_ahead(a.pf, a.sptr, cols_of<I>(a.cols), a.val64, s_, s1);
      double y[K];
      row_product<K, true, double>(a.sptr, cols_of<I>(a.cols), a.val64, a.diag64, s_, lane, act,
                                   g64, y);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        st_vec(a.t[k] + row_, y[k]);
        acc[2 * k] += y[k] * ld_ro(a.r[k] + row_);
        acc[2 * k + 1] += y[k] * y[k];
      }
    }
  } else if constexpr (!kMixed) {
    slice_rows<K, double, true, double, double, I>(n, a.sptr, cols_of<I>(a.cols), a.val64,
                                                   a.diag64, s0, s1, a.pf, act, g64, pre64,
                                                   post64);
  } else {
    slice_rows<K, float, false, float, double, I>(n, a.sptr, cols_of<I>(a.cols), a.val32, a.dc,
                                                  s0, s1, a.pf, act, g32, pre32, post32);
  }
  if (!last_block<2 * K>(acc, a.part, a.counter + 5, sm)) return;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      st->omega[k] = sm[2 * k] / sm[2 * k + 1];
      if (!isfinite(st->omega[k])) {
        st->active[k] = 0;
        st->status[k] = SFR_BREAKDOWN;
        st->iters[k] = st->j + 1;
      }
    }
  }
}

// B2: x += w z ; r -= w t ; (r, r), (r, r0) ; full-step test, beta
template <int K, bool kMixed>
__global__ void __launch_bounds__(256) k_bicg_b2(const SArgs<K> a, SState<K> *st) {
  SFR_SHARED_RED(2 * K);
  if (!st->any) return;
  const int n = a.n;
  int act[K];
  load_active<K>(st, act);
  double acc[2 * K], omv[K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
#pragma unroll
  for (int k = 0; k < K; ++k) omv[k] = st->omega[k];
  SFR_FOR_PAIRS(i) {
    const int r = 2 * i;
    const bool two = r + 1 < n;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      if (!kMixed) {
        const double w = omv[k];
        const double2 zv = ld2ro(a.z[k] + r), tv = ld2ro(a.t[k] + r), r0 = ld2ro(a.r0[k] + r);
        double2 xv = ld2(a.x[k] + r), rv = ld2(a.r[k] + r);
        xv.x = xadd(xv.x, xmul(w, zv.x));
        xv.y = xadd(xv.y, xmul(w, zv.y));
        rv.x = xsub(rv.x, xmul(w, tv.x));
        rv.y = xsub(rv.y, xmul(w, tv.y));
        st2(a.x[k] + r, xv);
        st2(a.r[k] + r, rv);
        acc[2 * k] += rv.x * rv.x;
        acc[2 * k + 1] += rv.x * r0.x;
        if (two) {
          acc[2 * k] += rv.y * rv.y;
          acc[2 * k + 1] += rv.y * r0.y;
        }
      } else {
        const float wf = static_cast<float>(omv[k]);
        const float2 zv = ld2ro(a.fz[k] + r), tv = ld2ro(a.ft[k] + r), r0 = ld2ro(a.fr0[k] + r);
        float2 xs = ld2(a.fxs[k] + r), rv = ld2(a.fr[k] + r);
        xs.x = fmaf(wf, zv.x, xs.x);
        xs.y = fmaf(wf, zv.y, xs.y);
        rv.x = fmaf(-wf, tv.x, rv.x);
        rv.y = fmaf(-wf, tv.y, rv.y);
        st2(a.fxs[k] + r, xs);
        st2(a.fr[k] + r, rv);
        acc[2 * k] += static_cast<double>(rv.x) * static_cast<double>(rv.x);
        acc[2 * k + 1] += static_cast<double>(rv.x) * static_cast<double>(r0.x);
        if (two) {
          acc[2 * k] += static_cast<double>(rv.y) * static_cast<double>(rv.y);
          acc[2 * k + 1] += static_cast<double>(rv.y) * static_cast<double>(r0.y);
        }
      }
    }
  }
  if (!last_block<2 * K>(acc, a.part, a.counter + 6, sm)) return;
  if (threadIdx.x == 0) {
    const unsigned j = st->j;
    int any = 0, any_upd = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      st->upd[k] = 0;
      if (!act[k]) continue;
      const double est = sqrt(sm[2 * k]);
      st->beta[k] = (sm[2 * k + 1] / st->rr0[k]) * (st->alpha[k] / st->omega[k]);
      if (!kMixed) {
        if (est < st->conv[k]) {
          st->active[k] = 0;
          st->iters[k] = j + 1;
        }
      } else if (est < st->conv[k] || est < st->call.delta * st->rmax[k]) {
        st->upd[k] = 1;
        any_upd = 1;
      }
      if (st->active[k] && !st->upd[k]) {
        if (!isfinite(st->beta[k])) {
          st->active[k] = 0;
          st->status[k] = SFR_BREAKDOWN;
          st->iters[k] = j + 1;
        } else if (j + 1 >= st->call.maxit) {
          st->active[k] = 0;
          st->status[k] = SFR_MAXIT;
          st->iters[k] = j + 2;
        }
      }
      any |= st->active[k];
    }
    // The refresh reads the FP64 matrix once for all right-hand sides, so
    // when one is due every other active one is refreshed in the same pass
    // (a reliable update is valid at any iteration).  Their later triggers
    // then tend to coincide, and fewer refresh passes are run in all.
    if (kMixed && K > 1 && any_upd) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (st->active[k]) st->upd[k] = 1;
    }
    st->j = j + 1;
    st->any = any;
    st->any_upd = any_upd;
    if (!any && a.in_graph) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// C: p = r + beta (p - w v) ; z = M p
template <int K, bool kMixed>
__global__ void __launch_bounds__(256) k_bicg_c(const SArgs<K> a, SState<K> *st) {
  if (!st->any) return;
  int act[K];
  load_active<K>(st, act);
  double bv[K], wv[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    bv[k] = st->beta[k];
    wv[k] = st->omega[k];
  }
  SFR_FOR_PAIRS(i) {
    const int r = 2 * i;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      if (!kMixed) {
        const double2 rv = ld2ro(a.r[k] + r), q = ld2ro(a.q[k] + r), m = ld2ro(a.m[k] + r);
        double2 p = ld2(a.p0[k] + r);
        p.x = xadd(rv.x, xmul(bv[k], xsub(p.x, xmul(wv[k], q.x))));
        p.y = xadd(rv.y, xmul(bv[k], xsub(p.y, xmul(wv[k], q.y))));
        st2(a.p0[k] + r, p);
        st2(a.z[k] + r, make_double2(xmul(p.x, m.x), xmul(p.y, m.y)));
      } else {
        const float bf = static_cast<float>(bv[k]);
        const float wf = static_cast<float>(wv[k]);
        const float2 rv = ld2ro(a.fr[k] + r), q = ld2ro(a.fq[k] + r), m = ld2ro(a.m32[k] + r);
        float2 p = ld2(a.fp0[k] + r);
        p.x = fmaf(bf, fmaf(-wf, q.x, p.x), rv.x);
        p.y = fmaf(bf, fmaf(-wf, q.y, p.y), rv.y);
        st2(a.fp0[k] + r, p);
        st2(a.fz[k] + r, make_float2(m.x * p.x, m.y * p.y));
      }
    }
  }
}

// ============================ host ======================================

struct GraphKey {
  int solver, k, precision, threads, spw;
  int shared_diag;  // the K right-hand sides share one diagonal
  int pf;           // SpMV-phase L2 prefetch distance
  int fused;        // FP64 PCG, one right-hand side: one cooperative kernel an iteration
  int staged;       // BiCGSTAB: SpMV phases with slices staged in shared memory
  bool operator<(const GraphKey &o) const {
    return std::tie(solver, k, precision, threads, spw, shared_diag, pf, fused, staged) <
           std::tie(o.solver, o.k, o.precision, o.threads, o.spw, o.shared_diag, o.pf, o.fused,
                    o.staged);
  }
};

// One instantiated graph with everything it touches: its own padded
// workspace, partials, counters, state and the by-value kernel arguments.
struct CachedGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *d_state = nullptr;  // SState<K>
  void *ws = nullptr;       // padded vectors
  double *part = nullptr;
  unsigned *counter = nullptr;
  std::vector<char> args;   // SArgs<K> (host copy, also baked into the nodes)
  cudaGraphConditionalHandle hwhile = 0;
  int grid_s = 0, grid_v = 0, threads = 256;
  int grid_o = 0;        // once-a-solve and refresh kernels: one wave of their own
  int grid_f = 0;        // fused iteration: co-resident blocks
  size_t smem_f = 0;     // fused iteration: dynamic shared memory a block
  unsigned long long *tagw = nullptr;  // fused modes 3-4: the broadcast word
  unsigned *ticks = nullptr;           // fused mode 4: update counts (inside tagw's allocation)
  size_t tag_bytes = 0;                // tagw's allocation
  bool staged = false;   // BiCGSTAB SpMV phases staged through shared memory
  size_t smem_s = 0;     // their dynamic shared memory a block
  uint64_t last_use = 0;
  int64_t bytes = 0;
};

struct EngineCache {
  std::map<GraphKey, std::unique_ptr<CachedGraph>> graphs;
  uint64_t clock = 0;
};
std::map<const sfr_system *, EngineCache> g_engines;
constexpr size_t kMaxGraphsPerSystem = 4;

cudaError_t add_kernel(cudaGraph_t g, cudaGraphNode_t *prev, void *func, int grid, int threads,
                       void **params, size_t smem = 0) {
  cudaKernelNodeParams p{};
  p.func = func;
  p.gridDim = dim3(grid);
  p.blockDim = dim3(threads);
  p.sharedMemBytes = static_cast<unsigned>(smem);
  p.kernelParams = params;
  cudaGraphNode_t node;
  cudaError_t e = cudaGraphAddKernelNode(&node, g, *prev ? prev : nullptr, *prev ? 1 : 0, &p);
  if (e == cudaSuccess) *prev = node;
  return e;
}

cudaError_t add_conditional(cudaGraph_t g, cudaGraphNode_t *prev, cudaGraphConditionalHandle h,
                            cudaGraphConditionalNodeType type, cudaGraph_t *body) {
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  cudaError_t e = cudaGraphAddNode(&node, g, *prev ? prev : nullptr, *prev ? 1 : 0, &p);
  if (e != cudaSuccess) return e;
  *body = p.conditional.phGraph_out[0];
  *prev = node;
  return cudaSuccess;
}

#define SFR_TRY(expr)                       \
  do {                                      \
    cudaError_t e_ = (expr);                \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

constexpr int kVecs64Plain = 11;  // diag b x m r z q p0 p1 r0 t
constexpr int kVecs64Mixed = 4;   // diag b x dc
constexpr int kVecs32 = 10;       // (unused) m32 r z q p0 p1 xs r0 t

inline int64_t padded(int n) { return (static_cast<int64_t>(n) + 3) & ~static_cast<int64_t>(3); }

// Stages a warp keeps in flight when BiCGSTAB's SpMV phases stage their
// slices through shared memory, and the widest slice (slots) they take.
constexpr int kStageDepth = 3;
constexpr int kStageMaxWidth = 8;

// BiCGSTAB's SpMV-phase kernels (A1, A2) of a graph.
template <int K, typename I>
void bicg_spmv_kernels(bool mixed, bool staged, const void **a1, const void **a2) {
  if constexpr (std::is_same<I, int16_t>::value) {
    if (staged) {
      *a1 = mixed ? (const void *)k_bicg_a1<K, true, I, kStageDepth>
                  : (const void *)k_bicg_a1<K, false, I, kStageDepth>;
      *a2 = mixed ? (const void *)k_bicg_a2<K, true, I, kStageDepth>
                  : (const void *)k_bicg_a2<K, false, I, kStageDepth>;
      return;
    }
  }
  *a1 = mixed ? (const void *)k_bicg_a1<K, true, I> : (const void *)k_bicg_a1<K, false, I>;
  *a2 = mixed ? (const void *)k_bicg_a2<K, true, I> : (const void *)k_bicg_a2<K, false, I>;
}

// Blocks of the iteration's SpMV kernel that fit on the GPU at once.
template <int K, typename I>
int resident_blocks(sfr_system *s, int solver, bool mixed, int threads, bool staged,
                    size_t smem) {
  const void *kern = nullptr, *unused = nullptr;
  if (solver == SFR_PCG)
    kern = mixed ? (const void *)k_pcg_a<K, true, I> : (const void *)k_pcg_a<K, false, I>;
  else
    bicg_spmv_kernels<K, I>(mixed, staged, &kern, &unused);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, staged ? smem : 0) !=
          cudaSuccess ||
      occ < 1)
    occ = 1;
  return occ * std::max(1, num_sms(s->device));
}

// spw > 0: `spw` slices per warp.  spw == 0: one wave, as many blocks as are
// resident at once (fewer for small systems), so no partial last wave leaves
// SMs idle while the phase's last blocks finish.
template <int K, typename I>
cudaError_t prepare(sfr_system *s, int solver, int precision, int threads, int spw,
                    int shared_diag, int pf, CachedGraph *cg) {
  const int n = s->n;
  const int64_t np = padded(n);
  const bool mixed = precision == SFR_MIXED;
  const int warps = threads / kWarp;
  cg->threads = threads;
  const int cap = s->A.max_width * kWarp;
  if (cg->staged) {
    cg->smem_s = static_cast<size_t>(warps) *
                 (mixed ? staged_warp_bytes<float, int16_t, kStageDepth>(cap)
                        : staged_warp_bytes<double, int16_t, kStageDepth>(cap));
    const void *k1 = nullptr, *k2 = nullptr;
    bicg_spmv_kernels<K, I>(mixed, true, &k1, &k2);
    SFR_TRY(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(cg->smem_s)));
    SFR_TRY(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(cg->smem_s)));
  }
  if (spw > 0)
    cg->grid_s = std::max(1, (s->A.nslices + warps * spw - 1) / (warps * spw));
  else
    cg->grid_s = std::max(
        1, std::min((s->A.nslices + warps - 1) / warps,
                    resident_blocks<K, I>(s, solver, mixed, threads, cg->staged, cg->smem_s)));
  {
    // start, refresh and post read the matrix like the SpMV phases but hold
    // more registers: one wave of their own, not the SpMV phase's grid
    const void *once[3] = {(const void *)k_post<K, I>,
                           solver == SFR_PCG
                               ? (mixed ? (const void *)k_pcg_start<K, true, I>
                                        : (const void *)k_pcg_start<K, false, I>)
                               : (mixed ? (const void *)k_bicg_start<K, true, I>
                                        : (const void *)k_bicg_start<K, false, I>),
                           solver == SFR_PCG ? (const void *)k_pcg_refresh<K, I>
                                             : (const void *)k_bicg_refresh<K, I>};
    int occ = 64;
    for (const void *k : once) {
      int o = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k, threads, 0) != cudaSuccess || o < 1)
        o = 1;
      occ = std::min(occ, o);
    }
    cg->grid_o = spw > 0 ? cg->grid_s
                         : std::max(1, std::min(cg->grid_s, occ * std::max(1, num_sms(s->device))));
  }
  const int npairs = (n + 1) / 2;
  const int wave = std::max(1, num_sms(s->device)) * (2048 / threads);
  cg->grid_v = std::max(1, std::min(wave, (npairs + threads - 1) / threads));
  const int gmax = std::max(cg->grid_s, cg->grid_v);
  const int n64 = mixed ? kVecs64Mixed : kVecs64Plain;
  const size_t bytes64 = sizeof(double) * static_cast<size_t>(np) * n64 * K;
  const size_t bytes32 = mixed ? sizeof(float) * static_cast<size_t>(np) * kVecs32 * K : 0;
  SFR_TRY(cudaMalloc(&cg->ws, bytes64 + bytes32));
  SFR_TRY(cudaMemset(cg->ws, 0, bytes64 + bytes32));  // padding rows stay finite
  SFR_TRY(cudaMalloc(&cg->d_state, sizeof(SState<K>)));
  SFR_TRY(cudaMalloc(&cg->part, sizeof(double) * kMaxNV * static_cast<size_t>(gmax)));
  SFR_TRY(cudaMalloc(&cg->counter, sizeof(unsigned) * kCounters));
  SFR_TRY(cudaMemset(cg->counter, 0, sizeof(unsigned) * kCounters));
  cg->bytes = static_cast<int64_t>(bytes64 + bytes32 + sizeof(double) * kMaxNV * gmax);

  cg->args.assign(sizeof(SArgs<K>), 0);
  SArgs<K> &a = *reinterpret_cast<SArgs<K> *>(cg->args.data());
  a.n = n;
  a.nslices = s->A.nslices;
  a.npairs = npairs;
  a.sptr = s->A.sptr;
  a.cols = SlotCols{s->A.col, s->A.off};
  a.val64 = s->A.val;
  a.val32 = s->A.val32;
  a.comp = s->d_comp;
  double *v64 = static_cast<double *>(cg->ws);
  float *v32 = reinterpret_cast<float *>(static_cast<char *>(cg->ws) + bytes64);
  for (int k = 0; k < K; ++k) {
    auto D = [&](int w) { return v64 + (static_cast<size_t>(w) * K + k) * np; };
    auto F = [&](int w) { return v32 + (static_cast<size_t>(w) * K + k) * np; };
    a.diag64[k] = D(0);
    a.b[k] = D(1);
    a.x[k] = D(2);
    if (mixed) {
      a.dc[k] = D(3);
      a.m32[k] = F(1);
      a.fr[k] = F(2);
      a.fz[k] = F(3);
      a.fq[k] = F(4);
      a.fp0[k] = F(5);
      a.fp1[k] = F(6);
      a.fxs[k] = F(7);
      a.fr0[k] = F(8);
      a.ft[k] = F(9);
    } else {
      a.m[k] = D(3);
      a.r[k] = D(4);
      a.z[k] = D(5);
      a.q[k] = D(6);
      a.p0[k] = D(7);
      a.p1[k] = D(8);
      a.r0[k] = D(9);
      a.t[k] = D(10);
    }
  }
  if (shared_diag) {
    for (int k = 1; k < K; ++k) {
      a.diag64[k] = a.diag64[0];
      if (mixed) {
        a.dc[k] = a.dc[0];
        a.m32[k] = a.m32[0];
      } else {
        a.m[k] = a.m[0];
      }
    }
  }
  a.shared_diag = shared_diag;
  a.pf = pf;
  a.stage_cap = cg->staged ? cap : 0;
  a.stage_err = reinterpret_cast<int *>(cg->counter + 15);
  a.part = cg->part;
  a.counter = cg->counter;
  return cudaSuccess;
}

// Launch shape of the fused PCG iteration: the most co-resident 256-thread
// blocks whose shared memory (8 bytes a row of the block's slices) still lets
// them all be resident at once.  0 when no shape fits.
template <typename I>
int fused_shape(sfr_system *s, int mode, size_t *smem) {
  const void *kern = fused_kernel<I>(mode);
  const int sms = std::max(1, num_sms(s->device));
  const int nsl = s->A.nslices;
  const int maxg = std::max(1, (nsl + 7) / 8);
  for (int per_sm = 8; per_sm >= 1; --per_sm) {
    const int G = std::min(maxg, per_sm * sms);
    const size_t bytes = static_cast<size_t>((nsl + G - 1) / G) * kWarp * sizeof(double);
    if (bytes > 200 * 1024) continue;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(bytes)) != cudaSuccess)
      continue;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, bytes) != cudaSuccess)
      continue;
    if (occ * sms >= G) {
      *smem = bytes;
      return G;
    }
  }
  return 0;
}

TagExchange fused_exchange(const CachedGraph *cg) {
  TagExchange t;
  t.word = cg->tagw;
  t.count = cg->counter + 11;
  t.err = reinterpret_cast<int *>(cg->counter + 14);
  t.spin_limit = 1u << 22;
  return t;
}

GridSync fused_barrier(const CachedGraph *cg) {
  GridSync g;
  g.count = cg->counter + 12;
  g.gen = cg->counter + 13;
  g.err = reinterpret_cast<int *>(cg->counter + 14);
  g.nblocks = static_cast<unsigned>(cg->grid_f);
  g.spin_limit = 1u << 22;
  return g;
}

// The graph for one (solver, K, precision, launch shape).
template <int K, typename I>
cudaError_t build_graph(sfr_system *s, int solver, int precision, int threads, int spw,
                        int shared_diag, int pf, int fused, CachedGraph *cg) {
  SFR_TRY((prepare<K, I>(s, solver, precision, threads, spw, shared_diag, pf, cg)));
  SFR_TRY(cudaGraphCreate(&cg->graph, 0));
  cudaGraph_t g = cg->graph;
  const bool mixed = precision == SFR_MIXED;
  SFR_TRY(cudaGraphConditionalHandleCreate(&cg->hwhile, g, 1, cudaGraphCondAssignDefault));
  SArgs<K> &a = *reinterpret_cast<SArgs<K> *>(cg->args.data());
  a.hwhile = cg->hwhile;
  a.in_graph = 1;

  // cudaGraphAddKernelNode copies the argument values these point to
  void *ps = cg->d_state;
  void *p2[2] = {&a, &ps};
  int stage1 = 1, stage2 = 2, zero = 0, one = 1;
  void *pf_sel[3] = {&a, &ps, &zero};
  void *pf_all[3] = {&a, &ps, &one};
  void *pr1[3] = {&a, &ps, &stage1};
  void *pr2[3] = {&a, &ps, &stage2};
  const int gs = cg->grid_s, gv = cg->grid_v, go = cg->grid_o;
  const void *a1k = nullptr, *a2k = nullptr;
  bicg_spmv_kernels<K, I>(mixed, cg->staged, &a1k, &a2k);
  const size_t ssm = cg->staged ? cg->smem_s : 0;

  cudaGraphNode_t prev = nullptr;
  {
    cudaMemsetParams mp{};
    mp.dst = cg->counter;
    mp.value = 0;
    mp.elementSize = sizeof(unsigned);
    mp.width = kCounters;
    mp.height = 1;
    mp.pitch = 0;
    SFR_TRY(cudaGraphAddMemsetNode(&prev, g, nullptr, 0, &mp));
  }
  if (fused >= 3 && cg->grid_f > 0) {
    // the fused iteration's exchange words (and mode 4's update counts, 64
    // bytes a block) start every solve at zero
    const size_t words = fused == 4 ? 16 + 16 * static_cast<size_t>(cg->grid_f) : 2;
    SFR_TRY(cudaMalloc(&cg->tagw, sizeof(unsigned) * words));
    cg->tag_bytes = sizeof(unsigned) * words;
    if (fused == 4) cg->ticks = reinterpret_cast<unsigned *>(cg->tagw) + 16;
    cudaMemsetParams mt{};
    mt.dst = cg->tagw;
    mt.value = 0;
    mt.elementSize = sizeof(unsigned);
    mt.width = words;
    mt.height = 1;
    mt.pitch = 0;
    cudaGraphNode_t mn;
    SFR_TRY(cudaGraphAddMemsetNode(&mn, g, &prev, 1, &mt));
    prev = mn;
  }
  cudaGraph_t body = nullptr;
  if (solver == SFR_PCG) {
    if (mixed) {
      SFR_TRY(add_kernel(g, &prev, (void *)k_setup<K, true>, gv, threads, p2));
      SFR_TRY(add_kernel(g, &prev, (void *)k_pcg_start<K, true, I>, go, threads, p2));
      SFR_TRY(add_conditional(g, &prev, cg->hwhile, cudaGraphCondTypeWhile, &body));
      cudaGraphNode_t bp = nullptr;
      SFR_TRY(add_kernel(body, &bp, (void *)k_pcg_a<K, true, I>, gs, threads, p2));
      SFR_TRY(add_kernel(body, &bp, (void *)k_pcg_b<K, true>, gv, threads, p2));
      // the reliable update as plain kernel nodes that return at once when
      // no right-hand side is due (a conditional IF node costs more than the
      // two empty launches)
      SFR_TRY(add_kernel(body, &bp, (void *)k_fold<K>, gv, threads, pf_sel));
      SFR_TRY(add_kernel(body, &bp, (void *)k_pcg_refresh<K, I>, go, threads, p2));
      SFR_TRY(add_kernel(body, &bp, (void *)k_pcg_c<K, true>, gv, threads, p2));
      SFR_TRY(add_kernel(g, &prev, (void *)k_fold<K>, gv, threads, pf_all));
    } else {
      SFR_TRY(add_kernel(g, &prev, (void *)k_setup<K, false>, gv, threads, p2));
      SFR_TRY(add_kernel(g, &prev, (void *)k_pcg_start<K, false, I>, go, threads, p2));
      SFR_TRY(add_conditional(g, &prev, cg->hwhile, cudaGraphCondTypeWhile, &body));
      cudaGraphNode_t bp = nullptr;
      if (fused && K == 1) {
        // one cooperative kernel an iteration (k_pcg_fused)
        GridSync gsync = fused_barrier(cg);
        TagExchange tx = fused_exchange(cg);
        unsigned *ticks = cg->ticks;
        void *pf3[5] = {&a, &ps, &gsync, &tx, &ticks};
        cudaKernelNodeParams kp{};
        kp.func = const_cast<void *>(fused_kernel<I>(fused));
        kp.gridDim = dim3(cg->grid_f);
        kp.blockDim = dim3(256);
        kp.sharedMemBytes = static_cast<unsigned>(cg->smem_f);
        kp.kernelParams = pf3;
        cudaGraphNode_t fn;
        SFR_TRY(cudaGraphAddKernelNode(&fn, body, nullptr, 0, &kp));
        cudaKernelNodeAttrValue coop{};
        coop.cooperative = 1;
        SFR_TRY(cudaGraphKernelNodeSetAttribute(fn, cudaLaunchAttributeCooperative, &coop));
      } else {
        SFR_TRY(add_kernel(body, &bp, (void *)k_pcg_a<K, false, I>, gs, threads, p2));
        SFR_TRY(add_kernel(body, &bp, (void *)k_pcg_b<K, false>, gv, threads, p2));
        SFR_TRY(add_kernel(body, &bp, (void *)k_pcg_c<K, false>, gv, threads, p2));
      }
    }
  } else {
    if (mixed) {
      SFR_TRY(add_kernel(g, &prev, (void *)k_setup<K, true>, gv, threads, p2));
      SFR_TRY(add_kernel(g, &prev, (void *)k_bicg_start<K, true, I>, go, threads, p2));
      SFR_TRY(add_conditional(g, &prev, cg->hwhile, cudaGraphCondTypeWhile, &body));
      cudaGraphNode_t bp = nullptr;
      SFR_TRY(add_kernel(body, &bp, const_cast<void *>(a1k), gs, threads, p2, ssm));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_b1<K, true>, gv, threads, p2));
      // the reliable updates as plain kernel nodes that return at once when
      // no right-hand side is due (as in the mixed PCG body)
      SFR_TRY(add_kernel(body, &bp, (void *)k_fold<K>, gv, threads, pf_sel));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_refresh<K, I>, go, threads, pr1));
      SFR_TRY(add_kernel(body, &bp, const_cast<void *>(a2k), gs, threads, p2, ssm));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_b2<K, true>, gv, threads, p2));
      SFR_TRY(add_kernel(body, &bp, (void *)k_fold<K>, gv, threads, pf_sel));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_refresh<K, I>, go, threads, pr2));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_c<K, true>, gv, threads, p2));
      SFR_TRY(add_kernel(g, &prev, (void *)k_fold<K>, gv, threads, pf_all));
    } else {
      SFR_TRY(add_kernel(g, &prev, (void *)k_setup<K, false>, gv, threads, p2));
      SFR_TRY(add_kernel(g, &prev, (void *)k_bicg_start<K, false, I>, go, threads, p2));
      SFR_TRY(add_conditional(g, &prev, cg->hwhile, cudaGraphCondTypeWhile, &body));
      cudaGraphNode_t bp = nullptr;
      SFR_TRY(add_kernel(body, &bp, const_cast<void *>(a1k), gs, threads, p2, ssm));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_b1<K, false>, gv, threads, p2));
      SFR_TRY(add_kernel(body, &bp, const_cast<void *>(a2k), gs, threads, p2, ssm));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_b2<K, false>, gv, threads, p2));
      SFR_TRY(add_kernel(body, &bp, (void *)k_bicg_c<K, false>, gv, threads, p2));
    }
  }
  SFR_TRY(add_kernel(g, &prev, (void *)k_post<K, I>, go, threads, p2));
  SFR_TRY(cudaGraphInstantiate(&cg->exec, g, 0));
  return cudaSuccess;
}

void free_graph(CachedGraph *cg) {
  if (cg->exec) cudaGraphExecDestroy(cg->exec);
  if (cg->graph) cudaGraphDestroy(cg->graph);
  cudaFree(cg->d_state);
  cudaFree(cg->ws);
  cudaFree(cg->part);
  cudaFree(cg->counter);
  cudaFree(cg->tagw);
  *cg = CachedGraph{};
}

// The same kernels launched from a host loop for `maxit` iterations (kernels
// of finished solves return at once).  For profilers, which cannot look into
// graphs with conditional nodes; never the production path.
template <int K, typename I>
cudaError_t launch_loop(CachedGraph *cg, int solver, bool mixed, int fused, uint32_t maxit,
                        cudaStream_t st) {
  SArgs<K> a = *reinterpret_cast<const SArgs<K> *>(cg->args.data());
  a.in_graph = 0;
  auto *ps = static_cast<SState<K> *>(cg->d_state);
  const int gs = cg->grid_s, gv = cg->grid_v, go = cg->grid_o, t = cg->threads;
  const void *a1k = nullptr, *a2k = nullptr;
  bicg_spmv_kernels<K, I>(mixed, cg->staged, &a1k, &a2k);
  const size_t ssm = cg->staged ? cg->smem_s : 0;
  void *pa[2] = {&a, &ps};
  SFR_TRY(cudaMemsetAsync(cg->counter, 0, sizeof(unsigned) * kCounters, st));
  if (cg->tagw) SFR_TRY(cudaMemsetAsync(cg->tagw, 0, cg->tag_bytes, st));
  if (solver == SFR_PCG) {
    if (mixed) {
      k_setup<K, true><<<gv, t, 0, st>>>(a, ps);
      k_pcg_start<K, true, I><<<go, t, 0, st>>>(a, ps);
      for (uint32_t it = 0; it < maxit; ++it) {
        k_pcg_a<K, true, I><<<gs, t, 0, st>>>(a, ps);
        k_pcg_b<K, true><<<gv, t, 0, st>>>(a, ps);
        k_fold<K><<<gv, t, 0, st>>>(a, ps, 0);
        k_pcg_refresh<K, I><<<go, t, 0, st>>>(a, ps);
        k_pcg_c<K, true><<<gv, t, 0, st>>>(a, ps);
      }
      k_fold<K><<<gv, t, 0, st>>>(a, ps, 1);
    } else {
      k_setup<K, false><<<gv, t, 0, st>>>(a, ps);
      k_pcg_start<K, false, I><<<go, t, 0, st>>>(a, ps);
      for (uint32_t it = 0; it < maxit; ++it) {
        if constexpr (K == 1) {
          if (fused) {
            GridSync gsync = fused_barrier(cg);
            TagExchange tx = fused_exchange(cg);
            unsigned *ticks = cg->ticks;
            void *pf3[5] = {&a, &ps, &gsync, &tx, &ticks};
            SFR_TRY(cudaLaunchCooperativeKernel(fused_kernel<I>(fused), dim3(cg->grid_f),
                                                dim3(256), pf3, cg->smem_f, st));
            if (fused == 4) break;  // the whole loop in one launch
            continue;
          }
        }
        k_pcg_a<K, false, I><<<gs, t, 0, st>>>(a, ps);
        k_pcg_b<K, false><<<gv, t, 0, st>>>(a, ps);
        k_pcg_c<K, false><<<gv, t, 0, st>>>(a, ps);
      }
    }
  } else {
    if (mixed) {
      k_setup<K, true><<<gv, t, 0, st>>>(a, ps);
      k_bicg_start<K, true, I><<<go, t, 0, st>>>(a, ps);
      for (uint32_t it = 0; it < maxit; ++it) {
        SFR_TRY(cudaLaunchKernel(a1k, dim3(gs), dim3(t), pa, ssm, st));
        k_bicg_b1<K, true><<<gv, t, 0, st>>>(a, ps);
        k_fold<K><<<gv, t, 0, st>>>(a, ps, 0);
        k_bicg_refresh<K, I><<<go, t, 0, st>>>(a, ps, 1);
        SFR_TRY(cudaLaunchKernel(a2k, dim3(gs), dim3(t), pa, ssm, st));
        k_bicg_b2<K, true><<<gv, t, 0, st>>>(a, ps);
        k_fold<K><<<gv, t, 0, st>>>(a, ps, 0);
        k_bicg_refresh<K, I><<<go, t, 0, st>>>(a, ps, 2);
        k_bicg_c<K, true><<<gv, t, 0, st>>>(a, ps);
      }
      k_fold<K><<<gv, t, 0, st>>>(a, ps, 1);
    } else {
      k_setup<K, false><<<gv, t, 0, st>>>(a, ps);
      k_bicg_start<K, false, I><<<go, t, 0, st>>>(a, ps);
      for (uint32_t it = 0; it < maxit; ++it) {
        SFR_TRY(cudaLaunchKernel(a1k, dim3(gs), dim3(t), pa, ssm, st));
        k_bicg_b1<K, false><<<gv, t, 0, st>>>(a, ps);
        SFR_TRY(cudaLaunchKernel(a2k, dim3(gs), dim3(t), pa, ssm, st));
        k_bicg_b2<K, false><<<gv, t, 0, st>>>(a, ps);
        k_bicg_c<K, false><<<gv, t, 0, st>>>(a, ps);
      }
    }
  }
  k_post<K, I><<<go, t, 0, st>>>(a, ps);
  return cudaGetLastError();
}

template <int K>
int run(sfr_system *s, int solver, const double *d_diag_k, const double *d_b, double *d_x,
        double tol, uint32_t maxit, int newx, int precision, double delta, int threads, int spw,
        int pf, int fused, bool loop, cudaStream_t st, SolveOut *out, float *ms) {
  const int n = s->n;
  if (maxit == 0) return SFR_BAD_INPUT;
  EngineCache &ec = g_engines[s];
  const int shared_diag = K > 1 && !d_diag_k ? 1 : 0;
  // the fused iteration serves FP64 PCG with one right-hand side when a
  // co-resident shape exists; other solves take the three-kernel iteration
  fused = K == 1 && solver == SFR_PCG && precision == SFR_FP64 ? fused : 0;
  size_t smem_f = 0;
  int grid_f = 0;
  if (fused)
    grid_f = s->A.off ? fused_shape<int16_t>(s, fused, &smem_f)
                      : fused_shape<int>(s, fused, &smem_f);
  if (fused && grid_f <= 0) fused = 0;
  // BiCGSTAB's SpMV phases stage their slices through shared memory when
  // the columns are 16-bit offsets and no slice is wider than a stage
  const int staged = solver != SFR_PCG && s->graph_stage && s->A.off &&
                             s->A.max_width <= kStageMaxWidth
                         ? 1
                         : 0;
  GraphKey key{solver, K, precision, threads, spw, shared_diag, pf, fused, staged};
  auto it = ec.graphs.find(key);
  if (it == ec.graphs.end()) {
    if (ec.graphs.size() >= kMaxGraphsPerSystem) {  // drop the least recently used
      auto lru = ec.graphs.begin();
      for (auto g = ec.graphs.begin(); g != ec.graphs.end(); ++g)
        if (g->second->last_use < lru->second->last_use) lru = g;
      free_graph(lru->second.get());
      ec.graphs.erase(lru);
    }
    auto cg = std::make_unique<CachedGraph>();
    cg->grid_f = grid_f;
    cg->smem_f = smem_f;
    cg->staged = staged != 0;
    const cudaError_t be =
        s->A.off ? build_graph<K, int16_t>(s, solver, precision, threads, spw, shared_diag, pf,
                                           fused, cg.get())
                 : build_graph<K, int>(s, solver, precision, threads, spw, shared_diag, pf,
                                       fused, cg.get());
    if (be != cudaSuccess) {
      set_last_error(cudaGetErrorString(be));
      free_graph(cg.get());
      return SFR_CUDA_ERROR;
    }
    it = ec.graphs.emplace(key, std::move(cg)).first;
  }
  CachedGraph *cg = it->second.get();
  cg->last_use = ++ec.clock;
  const SArgs<K> &a = *reinterpret_cast<const SArgs<K> *>(cg->args.data());
  const bool mixed = precision == SFR_MIXED;
  SCall call{tol, delta, maxit, newx};

  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  cudaError_t err = cudaSuccess;
  const size_t vb = sizeof(double) * static_cast<size_t>(n);
  for (int k = 0; k < K && err == cudaSuccess; ++k) {
    const double *dg = d_diag_k ? d_diag_k + static_cast<size_t>(k) * n : s->d_diag;
    if (k == 0 || !shared_diag)
      err = cudaMemcpyAsync(a.diag64[k], dg, vb, cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(a.b[k], d_b + static_cast<size_t>(k) * n, vb,
                            cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess && !newx)
      err = cudaMemcpyAsync(a.x[k], d_x + static_cast<size_t>(k) * n, vb,
                            cudaMemcpyDeviceToDevice, st);
  }
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(cg->d_state, &call, sizeof(call), cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess)
    err = !loop     ? cudaGraphLaunch(cg->exec, st)
          : s->A.off ? launch_loop<K, int16_t>(cg, solver, mixed, fused, maxit, st)
                     : launch_loop<K, int>(cg, solver, mixed, fused, maxit, st);
  for (int k = 0; k < K && err == cudaSuccess; ++k)
    err = cudaMemcpyAsync(d_x + static_cast<size_t>(k) * n, a.x[k], vb, cudaMemcpyDeviceToDevice,
                          st);
  cudaEventRecord(e1, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(out, static_cast<SState<K> *>(cg->d_state)->out, sizeof(SolveOut) * K,
                          cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) {
    set_last_error(cudaGetErrorString(err));
    return SFR_CUDA_ERROR;
  }
  return SFR_OK;
}

}  // namespace

int wait_selftest_fused(int32_t kind, int32_t absent, uint32_t spin_limit, cudaStream_t st) {
  constexpr int kGrid = 4;
  if ((kind != 0 && kind != 1) || absent < 0 || absent >= kGrid) return SFR_BAD_INPUT;
  // control words: grid_sync count, generation and error (0-2), the tagged
  // word (bytes 16-23), the exchange's arrivals (6), the block partials
  // (bytes 32-63)
  unsigned *ctl = nullptr;
  if (cudaMalloc(&ctl, 64) != cudaSuccess) return SFR_CUDA_ERROR;
  GridSync gs;
  gs.count = ctl;
  gs.gen = ctl + 1;
  gs.err = reinterpret_cast<int *>(ctl + 2);
  gs.nblocks = kGrid;
  gs.spin_limit = spin_limit;
  TagExchange tx;
  tx.word = reinterpret_cast<unsigned long long *>(ctl + 4);
  tx.count = ctl + 6;
  tx.err = gs.err;
  tx.spin_limit = spin_limit;
  double *part = reinterpret_cast<double *>(ctl + 8);
  void *params[] = {&kind, &absent, &gs, &tx, &part};
  int err = 0;
  cudaError_t ce = cudaMemsetAsync(ctl, 0, 64, st);
  if (ce == cudaSuccess)
    ce = cudaLaunchCooperativeKernel(reinterpret_cast<void *>(k_wait_selftest), dim3(kGrid),
                                     dim3(128), params, 0, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&err, gs.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  cudaFree(ctl);
  if (ce != cudaSuccess) {
    set_last_error(cudaGetErrorString(ce));
    return SFR_CUDA_ERROR;
  }
  return err;
}

int solve_stream(sfr_system *s, int32_t solver, int32_t k, const double *d_diag_k,
                 const double *d_b, double *d_x, double tol, uint32_t maxit, int32_t newx,
                 int32_t precision, double delta, int threads, int spw, int pf, int fused,
                 bool loop, cudaStream_t st, sfr_solve_info *info) {
  if (k < 1 || k > kMaxK) return SFR_BAD_INPUT;
  if (threads != 128 && threads != 256) return SFR_BAD_INPUT;
  if (spw < 0 || spw > 64) return SFR_BAD_INPUT;
  if (pf < 0 || pf > 8) return SFR_BAD_INPUT;
  SolveOut out[kMaxK];
  float ms = 0.f;
  int rc;
  switch (k) {
    case 1: rc = run<1>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, precision, delta, threads, spw, pf, fused, loop, st, out, &ms); break;
    case 2: rc = run<2>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, precision, delta, threads, spw, pf, fused, loop, st, out, &ms); break;
    case 3: rc = run<3>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, precision, delta, threads, spw, pf, fused, loop, st, out, &ms); break;
    default: rc = run<4>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, precision, delta, threads, spw, pf, fused, loop, st, out, &ms); break;
  }
  if (rc != SFR_OK) return rc;
  int worst = SFR_OK;
  for (int i = 0; i < k; ++i) {
    if (info) {
      sfr_solve_info &f = info[i];
      std::memset(&f, 0, sizeof(f));
      f.iters = out[i].iters;
      f.status = out[i].status;
      f.xKx = out[i].xKx;
      f.norm_x = out[i].norm_x;
      f.norm_r = out[i].norm_r;
      f.norm_r_m = out[i].norm_r_m;
      f.conv = out[i].conv;
      f.seconds = ms * 1e-3;
      f.refinements = out[i].refinements;
      f.inner_iters = out[i].inner_iters;
      f.relres = out[i].bnorm > 0 ? out[i].norm_r / out[i].bnorm : 0.0;
    }
    if (out[i].status != SFR_OK && worst == SFR_OK) worst = out[i].status;
  }
  return worst;
}

void release_stream_engine(const sfr_system *s) {
  auto it = g_engines.find(s);
  if (it == g_engines.end()) return;
  for (auto &kv : it->second.graphs) free_graph(kv.second.get());
  g_engines.erase(it);
}

}  // namespace sfr
