// Row-partitioned Jacobi-PCG and Jacobi-BiCGSTAB: the reference's MPI path
// (mpiPcg, Cg.c:256-442; mpiPbicgstab, Bicgstab.c:298-520) with one rank per
// GPU.
//
// Each rank holds its rows (nEqNov) and ghost entries (nEq - nEqNov) of every
// vector that a matrix-vector product reads.  Before each product the ghost
// entries are refreshed from their owners (comunicateNeq, ParallelMpi.c:3346):
// the owner packs the values its neighbours need into a send buffer and the
// exchange writes them into the receiver's ghost entries.  Each dot product is
// a rank-local sum followed by a sum over the ranks (the MPI_Allreduce of dot,
// HccaBlas.c:393-437).
//
// Transports.  An NCCL group (one rank per process) sends the halo with
// grouped ncclSend/ncclRecv straight into the receiver's ghost entries and
// sums with ncclAllReduce, all on the solve's stream.  A local group holds
// every rank in this process on one device: its halo is one gather kernel per
// rank reading the owner's vector, and its sums are taken in rank order by one
// small kernel.  Nothing waits on another kernel: the host orders the launches.
//
// Arithmetic is the reference's FP64 in its evaluation order (one rounding per
// multiply and add; matrix rows in the order mpiMatVecCsrD / mpiMatVecCsrDSym
// sum them).  A rank's partial dot is a fixed-order tree, so results agree
// with the reference to the summation-order spread, and every rank holds
// bit-identical Krylov scalars.
//
// Iterations are issued in chunks without a host round trip: every kernel
// returns at once after the solve has stopped (the stop is decided from the
// summed scalars, so all ranks decide alike), and the host reads the stop flag
// once a chunk.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace sfr {
void set_last_error(const char *msg);
}

namespace {

using sfr::xadd;
using sfr::xmul;
using sfr::xsub;

constexpr int kThreads = 256;
constexpr int kSlots = 8;  // sums per phase, at most
constexpr int kChunk = 32; // iterations per replay of the captured loop

// ---------------------------------------------------------------- NCCL ----
// Loaded at run time so that the library needs NCCL only when an NCCL group
// is made.
struct NcclApi {
  bool ok = false;
  std::string why;
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t,
                            ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t,
                       cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

NcclApi &nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    const char *env = std::getenv("SFR_NCCL_LIBRARY");
    void *h = dlopen(env && *env ? env : "libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      api.why = std::string("cannot load NCCL: ") + dlerror();
      return;
    }
    bool all = true;
    auto sym = [&](auto &fn, const char *name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
      all = all && fn != nullptr;
    };
    sym(api.GetUniqueId, "ncclGetUniqueId");
    sym(api.CommInitRank, "ncclCommInitRank");
    sym(api.CommDestroy, "ncclCommDestroy");
    sym(api.AllReduce, "ncclAllReduce");
    sym(api.Send, "ncclSend");
    sym(api.Recv, "ncclRecv");
    sym(api.GroupStart, "ncclGroupStart");
    sym(api.GroupEnd, "ncclGroupEnd");
    sym(api.GetErrorString, "ncclGetErrorString");
    if (!all) {
      api.why = "NCCL library lacks a required symbol";
      return;
    }
    api.ok = true;
  });
  return api;
}

// ------------------------------------------------------- device state ----
struct DState {
  double loc[kSlots];   // this rank's partial sums of the last phase
  double glob[kSlots];  // the sums over all ranks
  double conv, d, alpha, omega, rr0;
  int active, status, iters;
  unsigned j, maxit;
  double tol;
  int active_all;       // NCCL: the stop flag agreed over the ranks
};

struct Args {  // one rank's launch arguments
  int n, ncols, nslices;
  const int *sptr, *col;
  const double *val, *ad;
  const double *b;
  double *x, *m, *r, *z, *p, *q, *t, *v, *r0;
  double *part;
  unsigned *counter;
  DState *st;
  // local group: every rank's state, so that a kernel sums the ranks'
  // partials itself (in rank order); null for NCCL (the allreduce did it)
  DState *const *sts;
  int nranks;
};

// The sum over the ranks of partial s.
__device__ __forceinline__ double total(const Args &a, int s) {
  if (!a.sts) return a.st->glob[s];
  double t = a.sts[0]->loc[s];
  for (int r = 1; r < a.nranks; ++r) t = xadd(t, a.sts[r]->loc[s]);
  return t;
}

// Block partials of NV values -> the last block sums them in block order and
// returns true there, with the totals in tot (all its threads).
template <int NV>
__device__ bool rank_sums(const double (&acc)[NV], const Args &a, double (&tot)[NV]) {
  __shared__ double sm[32 * (NV + 1)];
  __shared__ bool s_last;
  sfr::block_partials<NV>(acc, a.part, gridDim.x, sm);
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(a.counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  sfr::grid_totals<NV>(a.part, gridDim.x, gridDim.x, tot, sm);
  if (threadIdx.x == 0) *a.counter = 0u;
  return true;
}

// y[row] of the rank's rows: diagonal product first, then the slots in order.
__device__ __forceinline__ double row_y(const Args &a, const double *xv, int row) {
  const int s = row >> 5, lane = row & 31;
  const int base = __ldg(a.sptr + s);
  const int w = (__ldg(a.sptr + s + 1) - base) >> 5;
  double y = xmul(sfr::ld_ro(a.ad + row), sfr::ld_vec(xv + row));
  const int *c = a.col + base + lane;
  const double *vv = a.val + base + lane;
  for (int e0 = 0; e0 < w; e0 += 6) {
    int jj[6];
    double av[6];
#pragma unroll
    for (int u = 0; u < 6; ++u)
      if (e0 + u < w) {
        jj[u] = sfr::ld_stream(c + (e0 + u) * 32);
        av[u] = sfr::ld_stream(vv + (e0 + u) * 32);
      }
#pragma unroll
    for (int u = 0; u < 6; ++u)
      if (e0 + u < w) y = xadd(y, xmul(av[u], sfr::ld_vec(xv + jj[u])));
  }
  return y;
}

#define ROWS_OF(a) \
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < (a).n; row += gridDim.x * blockDim.x)
// row pairs (2pr, 2pr+1) with 16-byte loads; every vector starts 16-byte
// aligned, and a last odd row is handled alone
#define PAIRS_OF(a) \
  for (int pr = blockIdx.x * blockDim.x + threadIdx.x; 2 * pr < (a).n; pr += gridDim.x * blockDim.x)

__device__ __forceinline__ double2 ld2(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ void st2(double *p, double2 v) { *reinterpret_cast<double2 *>(p) = v; }

__device__ __forceinline__ void stop(DState *st, int status, unsigned iters) {
  st->active = 0;
  st->status = status;
  st->iters = static_cast<int>(iters);
}

// ---- PCG (mpiPcg, Cg.c:256-442) ----------------------------------------
// m = 1/ad; x = 0 (newx, ghosts included); z = b m; sum (b, z)
__global__ void __launch_bounds__(kThreads) k_pcg_setup(Args a, int newx) {
  double acc[1] = {0.0};
  if (newx)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.ncols; i += gridDim.x * blockDim.x)
      a.x[i] = 0.0;
  ROWS_OF(a) {
    const double mi = 1.0 / a.ad[row];
    a.m[row] = mi;
    const double zi = xmul(a.b[row], mi);
    acc[0] = xadd(acc[0], xmul(a.b[row], zi));
  }
  double tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) a.st->loc[0] = tot[0];
}

// conv from the summed (b, M b); z = A x; r = b - z; z = M r; p = z; sum (r, z)
__global__ void __launch_bounds__(kThreads) k_pcg_start(Args a) {
  double acc[1] = {0.0};
  ROWS_OF(a) {
    const double y = row_y(a, a.x, row);
    const double ri = xsub(a.b[row], y);
    const double zi = xmul(ri, a.m[row]);
    a.r[row] = ri;
    a.z[row] = zi;
    a.p[row] = zi;
    acc[0] = xadd(acc[0], xmul(ri, zi));
  }
  double tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) {
    a.st->loc[1] = tot[0];
    a.st->conv = xmul(a.st->tol, sqrt(fabs(total(a, 0))));
  }
}

// d = the summed (r, z); z = A p; sum (z, p)
__global__ void __launch_bounds__(kThreads) k_pcg_a(Args a) {
  if (!a.st->active) return;
  double acc[1] = {0.0};
  ROWS_OF(a) {
    const double y = row_y(a, a.p, row);
    a.q[row] = y;
    acc[0] = xadd(acc[0], xmul(y, a.p[row]));
  }
  double tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) {
    a.st->loc[2] = tot[0];
    if (a.st->j == 0) a.st->d = total(a, 1);
  }
}

// alpha = d / (z, p); x += alpha p; r -= alpha z; z = M r; sum (r, z)
__global__ void __launch_bounds__(kThreads) k_pcg_b(Args a) {
  if (!a.st->active) return;
  const double alpha = a.st->d / total(a, 2);
  double acc[1] = {0.0};
  PAIRS_OF(a) {
    const int row = 2 * pr;
    if (row + 1 < a.n) {
      const double2 pv = ld2(a.p + row), qv = ld2(a.q + row), mv = ld2(a.m + row);
      double2 xv = ld2(a.x + row), rv = ld2(a.r + row), zv;
      xv.x = xadd(xv.x, xmul(alpha, pv.x));
      xv.y = xadd(xv.y, xmul(alpha, pv.y));
      rv.x = xsub(rv.x, xmul(alpha, qv.x));
      rv.y = xsub(rv.y, xmul(alpha, qv.y));
      zv.x = xmul(rv.x, mv.x);
      zv.y = xmul(rv.y, mv.y);
      st2(a.x + row, xv);
      st2(a.r + row, rv);
      st2(a.z + row, zv);
      acc[0] = xadd(acc[0], xmul(rv.x, zv.x));
      acc[0] = xadd(acc[0], xmul(rv.y, zv.y));
    } else {
      a.x[row] = xadd(a.x[row], xmul(alpha, a.p[row]));
      const double ri = xsub(a.r[row], xmul(alpha, a.q[row]));
      const double zi = xmul(ri, a.m[row]);
      a.r[row] = ri;
      a.z[row] = zi;
      acc[0] = xadd(acc[0], xmul(ri, zi));
    }
  }
  double tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) {
    a.st->loc[3] = tot[0];
    a.st->alpha = alpha;
  }
}

// beta = di / d; p = z + beta p; d = di; the stopping test sqrt|d| < conv
__global__ void __launch_bounds__(kThreads) k_pcg_c(Args a) {
  if (!a.st->active) return;
  const double di = total(a, 3);
  const double beta = di / a.st->d;
  const unsigned j = a.st->j;
  PAIRS_OF(a) {
    const int row = 2 * pr;
    if (row + 1 < a.n) {
      const double2 zv = ld2(a.z + row);
      double2 pv = ld2(a.p + row);
      pv.x = xadd(zv.x, xmul(beta, pv.x));
      pv.y = xadd(zv.y, xmul(beta, pv.y));
      st2(a.p + row, pv);
    } else {
      a.p[row] = xadd(a.z[row], xmul(beta, a.p[row]));
    }
  }
  double acc[1] = {0.0}, tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) {
    DState *st = a.st;
    st->d = di;
    st->j = j + 1;
    if (!isfinite(st->alpha) || !isfinite(beta)) stop(st, SFR_BREAKDOWN, j + 1);
    else if (sqrt(fabs(di)) < st->conv) stop(st, SFR_OK, j + 1);
    else if (j + 1 >= st->maxit) stop(st, SFR_MAXIT, j + 2);
  }
}

// post-processing (Cg.c:376-396): z = A x; (x, z), (x, x), r = b - z,
// (r, M r), (r, r); and (b, b) for the relative residual
__global__ void __launch_bounds__(kThreads) k_post(Args a, int pcg) {
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  ROWS_OF(a) {
    const double xi = a.x[row];
    const double y = row_y(a, a.x, row);
    acc[0] = xadd(acc[0], xmul(xi, y));
    acc[1] = xadd(acc[1], xmul(xi, xi));
    const double ri = xsub(a.b[row], y);
    acc[2] = xadd(acc[2], xmul(ri, pcg ? xmul(ri, a.m[row]) : 0.0));
    acc[3] = xadd(acc[3], xmul(ri, ri));
    acc[4] = xadd(acc[4], xmul(a.b[row], a.b[row]));
  }
  double tot[5];
  if (rank_sums<5>(acc, a, tot) && threadIdx.x == 0)
    for (int v = 0; v < 5; ++v) a.st->loc[v] = tot[v];
}

// ---- BiCGSTAB (mpiPbicgstab, Bicgstab.c:298-520) ------------------------
// m = 1/ad; x = 0 (newx); sum (b, b)
__global__ void __launch_bounds__(kThreads) k_bicg_setup(Args a, int newx) {
  double acc[1] = {0.0};
  if (newx)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.ncols; i += gridDim.x * blockDim.x)
      a.x[i] = 0.0;
  ROWS_OF(a) {
    a.m[row] = 1.0 / a.ad[row];
    acc[0] = xadd(acc[0], xmul(a.b[row], a.b[row]));
  }
  double tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) a.st->loc[0] = tot[0];
}

// conv = tol sqrt(b, b); z = A x; r0 = p = r = b - z; z = M p
__global__ void __launch_bounds__(kThreads) k_bicg_start(Args a) {
  ROWS_OF(a) {
    const double y = row_y(a, a.x, row);
    const double ri = xsub(a.b[row], y);
    a.r0[row] = ri;
    a.p[row] = ri;
    a.r[row] = ri;
    a.z[row] = xmul(ri, a.m[row]);
  }
  double acc[1] = {0.0}, tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0)
    a.st->conv = xmul(a.st->tol, sqrt(total(a, 0)));
}

// v = A z; sums (r, r0), (v, r0)
__global__ void __launch_bounds__(kThreads) k_bicg_a1(Args a) {
  if (!a.st->active) return;
  double acc[2] = {0.0, 0.0};
  ROWS_OF(a) {
    const double y = row_y(a, a.z, row);
    a.v[row] = y;
    const double r0i = a.r0[row];
    acc[0] = xadd(acc[0], xmul(a.r[row], r0i));
    acc[1] = xadd(acc[1], xmul(y, r0i));
  }
  double tot[2];
  if (rank_sums<2>(acc, a, tot) && threadIdx.x == 0) {
    a.st->loc[0] = tot[0];
    a.st->loc[1] = tot[1];
  }
}

// alpha = rr0 / (v, r0); x += alpha z; r -= alpha v; z = M r; sum (r, r)
__global__ void __launch_bounds__(kThreads) k_bicg_b1(Args a) {
  if (!a.st->active) return;
  const double rr0 = total(a, 0);
  const double alpha = rr0 / total(a, 1);
  double acc[1] = {0.0};
  ROWS_OF(a) {
    a.x[row] = xadd(a.x[row], xmul(alpha, a.z[row]));
    const double ri = xsub(a.r[row], xmul(alpha, a.v[row]));
    a.r[row] = ri;
    a.z[row] = xmul(ri, a.m[row]);
    acc[0] = xadd(acc[0], xmul(ri, ri));
  }
  double tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) {
    a.st->loc[2] = tot[0];
    a.st->alpha = alpha;
    a.st->rr0 = rr0;
  }
}

// the test sqrt(s, s) < conv; t = A z; sums (t, r), (t, t)
__global__ void __launch_bounds__(kThreads) k_bicg_a2(Args a) {
  if (!a.st->active) return;
  const double d = total(a, 2);
  const bool done = sqrt(d) < a.st->conv;
  double acc[2] = {0.0, 0.0};
  if (!done) {
    ROWS_OF(a) {
      const double y = row_y(a, a.z, row);
      a.t[row] = y;
      acc[0] = xadd(acc[0], xmul(y, a.r[row]));
      acc[1] = xadd(acc[1], xmul(y, y));
    }
  }
  double tot[2];
  if (rank_sums<2>(acc, a, tot) && threadIdx.x == 0) {
    DState *st = a.st;
    st->d = d;
    if (!isfinite(st->alpha)) stop(st, SFR_BREAKDOWN, st->j + 1);
    else if (done) stop(st, SFR_OK, st->j + 1);
    st->loc[3] = tot[0];
    st->loc[4] = tot[1];
  }
}

// w = (t, r) / (t, t); x += w z; r -= w t; sums (r, r), (r, r0)
__global__ void __launch_bounds__(kThreads) k_bicg_b2(Args a) {
  if (!a.st->active) return;
  const double w = total(a, 3) / total(a, 4);
  double acc[2] = {0.0, 0.0};
  ROWS_OF(a) {
    a.x[row] = xadd(a.x[row], xmul(w, a.z[row]));
    const double ri = xsub(a.r[row], xmul(w, a.t[row]));
    a.r[row] = ri;
    acc[0] = xadd(acc[0], xmul(ri, ri));
    acc[1] = xadd(acc[1], xmul(ri, a.r0[row]));
  }
  double tot[2];
  if (rank_sums<2>(acc, a, tot) && threadIdx.x == 0) {
    a.st->loc[5] = tot[0];
    a.st->loc[6] = tot[1];
    a.st->omega = w;
  }
}

// the test sqrt|r, r| < conv; beta = ((r, r0) / rr0) (alpha / w);
// p = r + beta (p - w v); z = M p
__global__ void __launch_bounds__(kThreads) k_bicg_c(Args a) {
  if (!a.st->active) return;
  const DState *cs = a.st;
  const double d = total(a, 5);
  const bool done = sqrt(fabs(d)) < cs->conv;
  const double w = cs->omega;
  const double beta = xmul(total(a, 6) / cs->rr0, cs->alpha / w);
  if (!done) {
    ROWS_OF(a) {
      const double pi = xadd(a.r[row], xmul(beta, xsub(a.p[row], xmul(w, a.v[row]))));
      a.p[row] = pi;
      a.z[row] = xmul(pi, a.m[row]);
    }
  }
  double acc[1] = {0.0}, tot[1];
  if (rank_sums<1>(acc, a, tot) && threadIdx.x == 0) {
    DState *st = a.st;
    const unsigned j = st->j;
    st->d = d;
    st->j = j + 1;
    if (done) stop(st, SFR_OK, j + 1);
    else if (!isfinite(w) || !isfinite(beta)) stop(st, SFR_BREAKDOWN, j + 1);
    else if (j + 1 >= st->maxit) stop(st, SFR_MAXIT, j + 2);
  }
}

// ---- halo ---------------------------------------------------------------
// send buffer: sbuf[i] = v[fmap_snd[i]]
// (every halo kernel returns at once after the solve stopped, unless `always`)
__global__ void k_pack(const double *v, const int *fmap_snd, int nsnd, double *sbuf,
                       const DState *st, int always) {
  if (!always && !st->active) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsnd; i += gridDim.x * blockDim.x)
    sbuf[i] = v[fmap_snd[i]];
}
// received values into their ghost entries (when they are not contiguous)
__global__ void k_unpack(double *v, const int *fmap_rcv, int nrcv, const double *rbuf,
                         const DState *st, int always) {
  if (!always && !st->active) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrcv; i += gridDim.x * blockDim.x)
    v[fmap_rcv[i]] = rbuf[i];
}
// local group: every rank's ghost entries of one vector, in one launch
// (*dst[i] = *src[i], the pairs listed once per vector)
__global__ void k_gather(double *const *dst, const double *const *src, int count,
                         const DState *st, int always) {
  if (!always && !st->active) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    *dst[i] = *src[i];
}
// local group: glob[s] of every rank = sum over the ranks in rank order of loc[s]
__global__ void k_rank_sum(DState *const *sts, int nranks, int first, int count, int always) {
  const int s = first + threadIdx.x;
  if (threadIdx.x >= count) return;
  if (!always && !sts[0]->active) return;
  double t = sts[0]->loc[s];
  for (int r = 1; r < nranks; ++r) t = xadd(t, sts[r]->loc[s]);
  for (int r = 0; r < nranks; ++r) sts[r]->glob[s] = t;
}
// values of the SELL slots from the raw al array
__global__ void k_gather_values(const int *src, long long nslots, const double *al, double *val) {
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nslots;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int s = src[e];
    val[e] = s >= 0 ? al[s] : 0.0;
  }
}

}  // namespace

// ------------------------------------------------------------ handles ----
struct sfr_dist_group {
  int kind = 0;  // 0 local, 1 NCCL
  int nranks = 0, rank = 0, device = 0;
  cudaStream_t stream = nullptr;
  std::vector<sfr_dist *> members;  // local: by rank
  bool wired = false;               // local: ghost sources built
  ncclComm_t comm = nullptr;
  // local: device table of each rank's state; per vector (x, p, z) the
  // ghost entries of every rank and their owners' entries
  DState **d_sts = nullptr;
  double **d_gdst[3] = {nullptr, nullptr, nullptr};
  double **d_gsrc[3] = {nullptr, nullptr, nullptr};
  int nghost = 0;
  int *h_flag = nullptr;      // pinned, two entries (read one chunk behind)
  // the iteration loop as a CUDA graph of kChunk iterations, per solver
  // (0 PCG, 1 BiCGSTAB), captured for the current set of ranks (epoch)
  cudaGraphExec_t chunk[2] = {nullptr, nullptr};
  uint64_t chunk_epoch[2] = {0, 0};
  uint64_t epoch = 1;
  cudaEvent_t flag_ev[2] = {nullptr, nullptr};
};

struct sfr_dist {
  sfr_dist_group *g = nullptr;
  int rank = 0, device = 0;
  int n = 0, ncols = 0, unsym = 0, nad = 0, nadr = 0, nsrc = 0;
  bool values_set = false;
  sfr::DevSell A;
  int64_t nslots = 0;
  double *d_raw = nullptr, *d_ad = nullptr;
  // interface
  int nrcv = 0, nsnd = 0;
  std::vector<int> viz, ia_rcv, ia_snd, fmap;
  bool rcv_contig = false;  // fMap[i] = nEqNov + i for the received values
  int *d_fmap = nullptr;    // nrcv + nsnd
  double *d_sbuf = nullptr, *d_rbuf = nullptr;
  // vectors (ncols each) and reductions
  double *d_vec = nullptr;
  double *x = nullptr, *b = nullptr, *m = nullptr, *r = nullptr, *z = nullptr, *p = nullptr,
         *q = nullptr, *t = nullptr, *v = nullptr, *r0 = nullptr;
  double *d_part = nullptr;
  unsigned *d_counter = nullptr;
  DState *d_st = nullptr;
  int max_blocks = 1;  // a resident wave of the widest kernel
};

namespace {

int fail(const std::string &msg, int code = SFR_BAD_INPUT) {
  sfr::set_last_error(msg.c_str());
  return code;
}
int cuda_fail(cudaError_t e, const char *where) {
  return fail(std::string(where) + ": " + cudaGetErrorString(e), SFR_CUDA_ERROR);
}
#define CK(call)                                            \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);     \
  } while (0)
#define NK(call)                                                                    \
  do {                                                                              \
    ncclResult_t r_ = (call);                                                       \
    if (r_ != ncclSuccess)                                                          \
      return fail(std::string(#call ": ") + nccl().GetErrorString(r_), SFR_CUDA_ERROR); \
  } while (0)

// One resident wave of `kernel` (its occupancy at kThreads a block), or
// fewer blocks when the rows do not need them.  A wave keeps the last-block
// counter at one arrival per resident block and leaves no tail.
template <typename K>
int wave_grid(K kernel, const sfr_dist *d) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> cache;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_pair(reinterpret_cast<const void *>(kernel), d->device);
    auto it = cache.find(key);
    if (it == cache.end()) {
      int occ = 0, sms = 148;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kThreads, 0);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device);
      it = cache.emplace(key, std::max(1, occ) * sms).first;
    }
    per_sm = it->second;
  }
  const int need = std::max(1, (d->n + kThreads - 1) / kThreads);
  return std::min({per_sm, need, d->max_blocks});
}

Args args_of(const sfr_dist *d) {
  Args a;
  a.n = d->n;
  a.ncols = d->ncols;
  a.nslices = d->A.nslices;
  a.sptr = d->A.sptr;
  a.col = d->A.col;
  a.val = d->A.val;
  a.ad = d->d_ad;
  a.b = d->b;
  a.x = d->x; a.m = d->m; a.r = d->r; a.z = d->z; a.p = d->p;
  a.q = d->q; a.t = d->t; a.v = d->v; a.r0 = d->r0;
  a.part = d->d_part;
  a.counter = d->d_counter;
  a.st = d->d_st;
  a.sts = d->g && d->g->kind == 0 ? d->g->d_sts : nullptr;
  a.nranks = d->g ? d->g->nranks : 1;
  return a;
}

void free_dist(sfr_dist *d) {
  if (!d) return;
  cudaSetDevice(d->device);
  sfr::free_sell(&d->A);
  cudaFree(d->d_raw);
  cudaFree(d->d_ad);
  cudaFree(d->d_fmap);
  cudaFree(d->d_sbuf);
  cudaFree(d->d_rbuf);
  cudaFree(d->d_vec);
  cudaFree(d->d_part);
  cudaFree(d->d_counter);
  cudaFree(d->d_st);
}

// Local group: pair every rank's receive lists with its neighbours' send
// lists and upload the ghost sources; the device tables of states and
// vectors.  Checks that the interfaces agree.
int wire_local(sfr_dist_group *g) {
  const int R = g->nranks;
  for (int r = 0; r < R; ++r)
    if (!g->members[r]) return fail("local group: rank " + std::to_string(r) + " not created");
  std::vector<double *> dst[3], src[3];
  for (int r = 0; r < R; ++r) {
    sfr_dist *d = g->members[r];
    for (size_t n = 0; n < d->viz.size(); ++n) {
      const int p = d->viz[n];
      const sfr_dist *o = g->members[p];
      const auto it = std::find(o->viz.begin(), o->viz.end(), r);
      const int len = d->ia_rcv[n + 1] - d->ia_rcv[n];
      if (it == o->viz.end()) {
        if (len == 0) continue;
        return fail("interface mismatch: rank " + std::to_string(p) + " does not list rank " +
                    std::to_string(r));
      }
      const size_t mm = static_cast<size_t>(it - o->viz.begin());
      const int slen = o->ia_snd[mm + 1] - o->ia_snd[mm];
      if (slen != len)
        return fail("interface mismatch: rank " + std::to_string(p) + " sends " +
                    std::to_string(slen) + " values to rank " + std::to_string(r) +
                    ", which receives " + std::to_string(len));
      for (int i = 0; i < len; ++i) {
        const int di = d->fmap[d->ia_rcv[n] + i];
        const int si = o->fmap[o->ia_snd[mm] + i];
        double *const dv[3] = {d->x, d->p, d->z};
        double *const sv[3] = {o->x, o->p, o->z};
        for (int w = 0; w < 3; ++w) {
          dst[w].push_back(dv[w] + di);
          src[w].push_back(sv[w] + si);
        }
      }
    }
  }
  for (int w = 0; w < 3; ++w) {
    cudaFree(g->d_gdst[w]);
    cudaFree(g->d_gsrc[w]);
    g->d_gdst[w] = g->d_gsrc[w] = nullptr;
  }
  g->nghost = static_cast<int>(dst[0].size());
  if (g->nghost > 0)
    for (int w = 0; w < 3; ++w) {
      const size_t bytes = dst[w].size() * sizeof(double *);
      CK(cudaMalloc(&g->d_gdst[w], bytes));
      CK(cudaMalloc(&g->d_gsrc[w], bytes));
      CK(cudaMemcpy(g->d_gdst[w], dst[w].data(), bytes, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(g->d_gsrc[w], src[w].data(), bytes, cudaMemcpyHostToDevice));
    }
  std::vector<DState *> sts(R);
  for (int r = 0; r < R; ++r) sts[r] = g->members[r]->d_st;
  CK(cudaMemcpy(g->d_sts, sts.data(), R * sizeof(DState *), cudaMemcpyHostToDevice));
  g->wired = true;
  ++g->epoch;
  return SFR_OK;
}

// Ghost entries of vector `which` (0 x, 1 p, 2 z) of every rank of this process.
int exchange(sfr_dist_group *g, sfr_dist *const *parts, int nlocal, int which, bool always) {
  const int aw = always ? 1 : 0;
  cudaStream_t st = g->stream;
  if (g->kind == 0) {
    if (g->nghost == 0) return SFR_OK;
    const int blocks = std::min(1184, (g->nghost + 255) / 256);
    k_gather<<<blocks, 256, 0, st>>>(g->d_gdst[which], g->d_gsrc[which], g->nghost,
                                     parts[0]->d_st, aw);
    CK(cudaGetLastError());
    return SFR_OK;
  }
  sfr_dist *d = parts[0];
  if (d->viz.empty()) return SFR_OK;
  double *v = which == 0 ? d->x : which == 1 ? d->p : d->z;
  if (d->nsnd > 0) {
    const int blocks = std::min(1184, (d->nsnd + 255) / 256);
    k_pack<<<blocks, 256, 0, st>>>(v, d->d_fmap + d->nrcv, d->nsnd, d->d_sbuf, d->d_st, aw);
    CK(cudaGetLastError());
  }
  double *rdst = d->rcv_contig ? v + d->n : d->d_rbuf;
  const NcclApi &api = nccl();
  NK(api.GroupStart());
  for (size_t n = 0; n < d->viz.size(); ++n) {
    const int peer = d->viz[n];
    const int slen = d->ia_snd[n + 1] - d->ia_snd[n];
    const int rlen = d->ia_rcv[n + 1] - d->ia_rcv[n];
    if (slen > 0)
      NK(api.Send(d->d_sbuf + (d->ia_snd[n] - d->nrcv), slen, ncclDouble, peer, g->comm, st));
    if (rlen > 0) NK(api.Recv(rdst + d->ia_rcv[n], rlen, ncclDouble, peer, g->comm, st));
  }
  NK(api.GroupEnd());
  if (!d->rcv_contig && d->nrcv > 0) {
    const int blocks = std::min(1184, (d->nrcv + 255) / 256);
    k_unpack<<<blocks, 256, 0, st>>>(v, d->d_fmap, d->nrcv, d->d_rbuf, d->d_st, aw);
    CK(cudaGetLastError());
  }
  return SFR_OK;
}

// glob[first..first+count) = the sums over the ranks of loc[...].  A local
// group's kernels sum the ranks' partials themselves; it runs the kernel only
// for the totals the host reads (`always`).
int rank_sum(sfr_dist_group *g, sfr_dist *const *parts, int first, int count, bool always) {
  if (g->kind == 0) {
    if (!always) return SFR_OK;
    k_rank_sum<<<1, 32, 0, g->stream>>>(g->d_sts, g->nranks, first, count, always ? 1 : 0);
    CK(cudaGetLastError());
    return SFR_OK;
  }
  DState *s = parts[0]->d_st;
  NK(nccl().AllReduce(s->loc + first, s->glob + first, count, ncclDouble, ncclSum, g->comm,
                      g->stream));
  return SFR_OK;
}

}  // namespace

extern "C" {

int sfr_dist_group_local(int32_t nparts, int32_t device, sfr_dist_group **out) {
  if (!out || nparts <= 0 || nparts > 32767) return fail("bad local group arguments");
  *out = nullptr;
  CK(cudaSetDevice(device));
  auto *g = new (std::nothrow) sfr_dist_group;
  if (!g) return fail("out of host memory");
  g->kind = 0;
  g->nranks = nparts;
  g->device = device;
  g->members.assign(nparts, nullptr);
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_sts, nparts * sizeof(DState *));
  if (e == cudaSuccess) e = cudaMallocHost(&g->h_flag, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->flag_ev[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->flag_ev[1], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    sfr_dist_group_destroy(g);
    return cuda_fail(e, "local group allocation");
  }
  *out = g;
  return SFR_OK;
}

int sfr_dist_nccl_id(uint8_t id[128]) {
  if (!id) return fail("id is NULL");
  NcclApi &api = nccl();
  if (!api.ok) return fail(api.why, SFR_UNSUPPORTED);
  ncclUniqueId u;
  NK(api.GetUniqueId(&u));
  static_assert(sizeof(u) == 128, "NCCL unique id is 128 bytes");
  std::memcpy(id, &u, 128);
  return SFR_OK;
}

int sfr_dist_group_nccl(int32_t nranks, int32_t rank, const uint8_t id[128], int32_t device,
                        sfr_dist_group **out) {
  if (!out || !id || nranks <= 0 || rank < 0 || rank >= nranks)
    return fail("bad NCCL group arguments");
  *out = nullptr;
  NcclApi &api = nccl();
  if (!api.ok) return fail(api.why, SFR_UNSUPPORTED);
  CK(cudaSetDevice(device));
  auto *g = new (std::nothrow) sfr_dist_group;
  if (!g) return fail("out of host memory");
  g->kind = 1;
  g->nranks = nranks;
  g->rank = rank;
  g->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocHost(&g->h_flag, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->flag_ev[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->flag_ev[1], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    sfr_dist_group_destroy(g);
    return cuda_fail(e, "NCCL group allocation");
  }
  ncclUniqueId u;
  std::memcpy(&u, id, 128);
  const ncclResult_t r = api.CommInitRank(&g->comm, nranks, u, rank);
  if (r != ncclSuccess) {
    g->comm = nullptr;
    sfr_dist_group_destroy(g);
    return fail(std::string("ncclCommInitRank: ") + api.GetErrorString(r), SFR_CUDA_ERROR);
  }
  *out = g;
  return SFR_OK;
}

int sfr_dist_group_destroy(sfr_dist_group *g) {
  if (!g) return SFR_OK;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->comm) nccl().CommDestroy(g->comm);
  for (sfr_dist *d : g->members)
    if (d) d->g = nullptr;
  cudaFree(g->d_sts);
  for (int w = 0; w < 3; ++w) {
    cudaFree(g->d_gdst[w]);
    cudaFree(g->d_gsrc[w]);
  }
  if (g->h_flag) cudaFreeHost(g->h_flag);
  for (int k = 0; k < 2; ++k) {
    if (g->chunk[k]) cudaGraphExecDestroy(g->chunk[k]);
    if (g->flag_ev[k]) cudaEventDestroy(g->flag_ev[k]);
  }
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return SFR_OK;
}

int sfr_dist_group_info(const sfr_dist_group *g, int32_t *kind, int32_t *nranks, int32_t *rank) {
  if (!g) return fail("group is NULL");
  if (kind) *kind = g->kind;
  if (nranks) *nranks = g->nranks;
  if (rank) *rank = g->rank;
  return SFR_OK;
}

int sfr_gpu_dist_create(sfr_dist_group *g, int32_t rank, int32_t nEq, int32_t nEqNov,
                        int32_t nAd, int32_t nAdR, const int32_t *ia, const int32_t *ja,
                        int32_t unsym, const sfr_interface *iNeq, sfr_dist **out) {
  return sfr_gpu_dist_create_storage(g, rank, SFR_CSRD, nEq, nEqNov, nAd, nAdR, ia, ja, unsym,
                                     iNeq, out);
}

int sfr_gpu_dist_create_storage(sfr_dist_group *g, int32_t rank, int32_t storage, int32_t nEq,
                                int32_t nEqNov, int32_t nAd, int32_t nAdR, const int32_t *ia,
                                const int32_t *ja, int32_t unsym, const sfr_interface *iNeq,
                                sfr_dist **out) {
  if (!out) return fail("out is NULL");
  *out = nullptr;
  if (!g || !ia || !iNeq) return fail("group, ia or iNeq is NULL");
  if (g->kind == 0 ? (rank < 0 || rank >= g->nranks) : rank != g->rank)
    return fail("rank does not belong to this group in this process");
  if (g->kind == 0 && g->members[rank]) return fail("rank already created in this group");
  if (nEqNov <= 0 || nEq < nEqNov || nAd < 0 || nAdR < 0) return fail("bad sizes");
  const bool coo = storage == SFR_CSRDCOO || storage == SFR_CSRCCOO;
  if (storage != SFR_CSRD && storage != SFR_CSRC && storage != SFR_ELLPACK && !coo)
    return fail("storage must be CSRD, CSRC, ELLPACK, CSRDCOO or CSRCCOO", SFR_UNSUPPORTED);
  if (storage == SFR_CSRDCOO && unsym)
    return fail("CSRDCOO is symmetric storage (Datastruct.c:199)", SFR_UNSUPPORTED);
  if (storage == SFR_CSRD && unsym && nAdR != 0)
    return fail("unsymmetric CSRD keeps ghost columns in its rows: nAdR must be 0");
  const int nghost = nEq - nEqNov;
  if (iNeq->nRcvs > nghost) return fail("nRcvs exceeds the ghost count");
  const int nviz = iNeq->nVizPart;
  const int nrcv = iNeq->nRcvs, nsnd = iNeq->nSends;
  if (nrcv < 0 || nsnd < 0) return fail("negative interface sizes");
  if (nviz > 0 && (!iNeq->iaSends || !iNeq->iaRcvs || !iNeq->vizPart))
    return fail("interface arrays are NULL");
  if (nrcv + nsnd > 0 && !iNeq->fMap) return fail("fMap is NULL");
  // interface checks
  std::vector<int> viz(nviz), iar(nviz + 1, 0), ias(nviz + 1, nrcv), fmap(nrcv + nsnd);
  for (int n = 0; n < nviz; ++n) {
    viz[n] = iNeq->vizPart[n];
    if (viz[n] < 0 || viz[n] >= g->nranks || viz[n] == rank)
      return fail("vizPart lists a rank outside the group or this rank");
  }
  if (nviz > 0) {
    for (int n = 0; n <= nviz; ++n) {
      iar[n] = iNeq->iaRcvs[n];
      ias[n] = iNeq->iaSends[n];
    }
    if (iar[0] != 0 || iar[nviz] != nrcv || ias[0] != nrcv || ias[nviz] != nrcv + nsnd)
      return fail("iaRcvs must run from 0 to nRcvs and iaSends from nRcvs to nRcvs+nSends");
    for (int n = 0; n < nviz; ++n)
      if (iar[n + 1] < iar[n] || ias[n + 1] < ias[n]) return fail("iaRcvs/iaSends not monotone");
  } else if (nrcv + nsnd != 0) {
    return fail("values to exchange without neighbours");
  }
  bool contig = true;
  for (int i = 0; i < nrcv + nsnd; ++i) {
    fmap[i] = iNeq->fMap[i];
    if (i < nrcv) {
      if (fmap[i] < nEqNov || fmap[i] >= nEq) return fail("a received value is not a ghost entry");
      contig = contig && fmap[i] == nEqNov + i;
    } else if (fmap[i] < 0 || fmap[i] >= nEqNov) {
      return fail("a sent value is not an owned entry");
    }
  }
  // the rows (columns local, ghosts included), in the reference's order
  const int ncols = nEq;
  std::vector<int64_t> ptr(nEqNov + 1, 0);
  std::vector<int32_t> col, src;
  int64_t nsrc = 0;
  if (storage == SFR_ELLPACK) {
    // ia = {width, nEqNov * width}; ja and the values row-major, every slot
    // in order, padded slots included (mpiMatVecEllPack, HccaBlas.c:5094)
    const int width = ia[0];
    if (width <= 0 || ia[1] != static_cast<int64_t>(nEqNov) * width)
      return fail("ELLPACK ia must be {width, nEqNov * width}");
    if (!ja) return fail("ja is NULL");
    nsrc = static_cast<int64_t>(nEqNov) * width;
    for (int64_t k = 0; k < nsrc; ++k)
      if (ja[k] < 0 || ja[k] >= ncols) return fail("ja out of range");
    col.assign(ja, ja + nsrc);
    src.resize(nsrc);
    for (int64_t k = 0; k < nsrc; ++k) src[k] = static_cast<int32_t>(k);
    for (int i = 0; i <= nEqNov; ++i) ptr[i] = static_cast<int64_t>(i) * width;
  } else {
    const int32_t base = ia[0];
    if (base != 0) return fail("ia[0] must be 0");
    for (int i = 0; i < nEqNov; ++i)
      if (ia[i + 1] < ia[i]) return fail("ia not monotone");
    if (ia[nEqNov] != nAd) return fail("ia[nEqNov] != nAd");
    const bool full_rows = storage == SFR_CSRD && unsym;
    // the rectangular (ghost-column) part: CSR at ia + nEqNov + 1; COO rows
    // at ia + 2 (nEqNov + 1) (Datastruct.c:129-260, 336-420)
    const int32_t *iar_m = full_rows ? nullptr : ia + nEqNov + 1;
    const int32_t *coo_row = coo ? ia + 2 * (nEqNov + 1) : nullptr;
    if (!full_rows) {
      if (iar_m[0] != 0) return fail("the rectangular part's ia must start at 0");
      for (int i = 0; i < nEqNov; ++i)
        if (iar_m[i + 1] < iar_m[i]) return fail("rectangular ia not monotone");
      if (iar_m[nEqNov] != nAdR) return fail("rectangular ia[nEqNov] != nAdR");
      if (coo)
        for (int i = 0; i < nEqNov; ++i)
          for (int k = iar_m[i]; k < iar_m[i + 1]; ++k)
            if (coo_row[k] != i) return fail("COO rows disagree with the rectangular ia");
    }
    if (nAd + nAdR > 0 && !ja) return fail("ja is NULL");
    for (int k = 0; k < nAd + nAdR; ++k)
      if (ja[k] < 0 || ja[k] >= ncols) return fail("ja out of range");
    if (full_rows) {
      nsrc = nAd;
      col.assign(ja, ja + nAd);
      src.resize(nAd);
      for (int k = 0; k < nAd; ++k) src[k] = k;
      for (int i = 0; i <= nEqNov; ++i) ptr[i] = ia[i];
    } else {
      // strict-lower square part + mirrored entries of later rows + ghost
      // columns.  The mirrored value is al[k] (symmetric) or au[k] = a[nAd+k]
      // (CSRC unsymmetric); the ghost values follow the square part's.
      // Order of a row (the reference's accumulation):
      //   CSR ghosts (mpiMatVecCsrDSym HccaBlas.c:2872-2890, mpiMatVecCsrC
      //   :4394): own lower entries, own ghost columns, mirrored entries;
      //   COO ghosts (mpiMatVecCsrDcooSym :2928, mpiMatVecCsrCcoo :4611):
      //   own lower entries, mirrored entries, then the ghost terms, which
      //   the reference adds after every row, in COO order.
      const bool split = storage == SFR_CSRC || storage == SFR_CSRCCOO;
      const int64_t mirror_off = split && unsym ? nAd : 0;
      const int64_t rect_off = split && unsym ? 2 * static_cast<int64_t>(nAd) : nAd;
      nsrc = rect_off + nAdR;
      for (int i = 0; i < nEqNov; ++i)
        for (int k = ia[i]; k < ia[i + 1]; ++k)
          if (ja[k] >= i) return fail("square part not strictly lower");
      std::vector<int64_t> up(nEqNov + 1, 0);
      for (int k = 0; k < nAd; ++k) ++up[ja[k] + 1];
      for (int i = 0; i < nEqNov; ++i) up[i + 1] += up[i];
      std::vector<int32_t> upc(nAd), ups(nAd);
      std::vector<int64_t> fill(up.begin(), up.end() - 1);
      for (int i = 0; i < nEqNov; ++i)
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
          const int64_t q = fill[ja[k]]++;
          upc[q] = i;
          ups[q] = k;
        }
      for (int i = 0; i < nEqNov; ++i) {
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
          col.push_back(ja[k]);
          src.push_back(k);
        }
        auto ghosts = [&]() -> bool {
          for (int k = iar_m[i]; k < iar_m[i + 1]; ++k) {
            if (ja[nAd + k] < nEqNov) return false;
            col.push_back(ja[nAd + k]);
            src.push_back(static_cast<int32_t>(rect_off + k));
          }
          return true;
        };
        if (!coo && !ghosts()) return fail("rectangular part names an owned column");
        for (int64_t u = up[i]; u < up[i + 1]; ++u) {
          col.push_back(upc[u]);
          src.push_back(static_cast<int32_t>(mirror_off + ups[u]));
        }
        if (coo && !ghosts()) return fail("rectangular part names an owned column");
        ptr[i + 1] = static_cast<int64_t>(col.size());
      }
    }
  }
  if (nsrc > INT32_MAX) return fail("too many values");
  // SELL-32 of the rows
  sfr::HostSell h;
  h.n = nEqNov;
  h.nslices = (nEqNov + 31) / 32;
  h.sptr.assign(h.nslices + 1, 0);
  int64_t total = 0;
  for (int s = 0; s < h.nslices; ++s) {
    int64_t w = 0;
    for (int l = 0; l < 32; ++l) {
      const int r = s * 32 + l;
      if (r < nEqNov) w = std::max<int64_t>(w, ptr[r + 1] - ptr[r]);
    }
    total += w * 32;
    if (total > INT32_MAX) return fail("too many slots");
    h.sptr[s + 1] = static_cast<int32_t>(total);
  }
  h.col.assign(total, 0);
  h.src.assign(total, -1);
  for (int s = 0; s < h.nslices; ++s) {
    const int w = (h.sptr[s + 1] - h.sptr[s]) / 32;
    for (int l = 0; l < 32; ++l) {
      const int r = s * 32 + l;
      const int64_t len = r < nEqNov ? ptr[r + 1] - ptr[r] : 0;
      for (int k = 0; k < w; ++k) {
        const int64_t e = h.sptr[s] + static_cast<int64_t>(k) * 32 + l;
        if (k < len) {
          h.col[e] = col[ptr[r] + k];
          h.src[e] = src[ptr[r] + k];
        } else {
          h.col[e] = r < nEqNov ? r : 0;
        }
      }
    }
  }
  h.nnz = static_cast<int64_t>(col.size());
  h.bandwidth = INT32_MAX;  // ghost columns: absolute indices, no 16-bit offsets

  CK(cudaSetDevice(g->device));
  auto *d = new (std::nothrow) sfr_dist;
  if (!d) return fail("out of host memory");
  d->g = g;
  d->rank = rank;
  d->device = g->device;
  d->n = nEqNov;
  d->ncols = ncols;
  d->unsym = unsym ? 1 : 0;
  d->nad = nAd;
  d->nadr = nAdR;
  d->nsrc = static_cast<int>(nsrc);
  d->nslots = total;
  d->nrcv = nrcv;
  d->nsnd = nsnd;
  d->viz = viz;
  d->ia_rcv = iar;
  d->ia_snd = ias;
  d->fmap = fmap;
  d->rcv_contig = contig;
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    d->max_blocks = sms * (2048 / kThreads);
  }
  int64_t bytes = 0;
  int rc = sfr::upload_sell(h, &d->A, &bytes);
  cudaError_t e = rc == SFR_OK ? cudaSuccess : cudaErrorMemoryAllocation;
  // vectors padded to an even length: each starts 16-byte aligned
  const size_t nv = (static_cast<size_t>(ncols) + 2) & ~static_cast<size_t>(1);
  if (e == cudaSuccess) e = cudaMalloc(&d->A.val, std::max<int64_t>(total, 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d->d_raw, std::max(d->nsrc, 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d->d_ad, nEqNov * sizeof(double));
  if (e == cudaSuccess && nrcv + nsnd > 0) {
    e = cudaMalloc(&d->d_fmap, (nrcv + nsnd) * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(d->d_fmap, fmap.data(), (nrcv + nsnd) * sizeof(int), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&d->d_sbuf, std::max(nsnd, 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d->d_rbuf, std::max(nrcv, 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d->d_vec, 10 * nv * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(d->d_vec, 0, 10 * nv * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d->d_part, static_cast<size_t>(d->max_blocks) * kSlots * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d->d_counter, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(d->d_counter, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&d->d_st, sizeof(DState));
  if (e == cudaSuccess) e = cudaMemset(d->d_st, 0, sizeof(DState));
  if (e != cudaSuccess) {
    free_dist(d);
    delete d;
    return rc != SFR_OK ? rc : cuda_fail(e, "partition allocation");
  }
  double *vv[10];
  for (int k = 0; k < 10; ++k) vv[k] = d->d_vec + k * nv;
  d->x = vv[0]; d->b = vv[1]; d->m = vv[2]; d->r = vv[3]; d->z = vv[4];
  d->p = vv[5]; d->q = vv[6]; d->t = vv[7]; d->v = vv[8]; d->r0 = vv[9];
  if (g->kind == 0) {
    g->members[rank] = d;
    g->wired = false;
  } else {
    g->members.assign(1, d);
  }
  ++g->epoch;
  *out = d;
  return SFR_OK;
}

int sfr_gpu_dist_set_values(sfr_dist *d, const double *al, const double *ad) {
  if (!d || !ad || (d->nsrc > 0 && !al)) return fail("NULL argument");
  CK(cudaSetDevice(d->device));
  if (d->nsrc > 0) CK(cudaMemcpy(d->d_raw, al, d->nsrc * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d->d_ad, ad, d->n * sizeof(double), cudaMemcpyHostToDevice));
  if (d->nslots > 0) {
    const int blocks = static_cast<int>(std::min<int64_t>(4096, (d->nslots + 255) / 256));
    k_gather_values<<<blocks, 256>>>(d->A.src, d->nslots, d->d_raw, d->A.val);
    CK(cudaGetLastError());
  }
  CK(cudaDeviceSynchronize());
  d->values_set = true;
  return SFR_OK;
}

int sfr_gpu_dist_solve(sfr_dist_group *g, int32_t nlocal, sfr_dist *const *parts,
                       int32_t solver, const double *const *b, double *const *x, double tol,
                       uint32_t maxIt, int32_t newX, sfr_solve_info *info) {
  if (!g || !parts || !b || !x) return fail("NULL argument");
  if (g->kind == 0 ? nlocal != g->nranks : nlocal != 1)
    return fail("pass every rank of a local group, or the one rank of an NCCL group");
  for (int k = 0; k < nlocal; ++k) {
    if (!parts[k] || parts[k]->g != g) return fail("a partition does not belong to this group");
    if (g->kind == 0 && parts[k]->rank != k) return fail("partitions must be in rank order");
    if (!parts[k]->values_set) return fail("values not set");
    if (!b[k] || !x[k]) return fail("b or x is NULL");
  }
  CK(cudaSetDevice(g->device));
  cudaStream_t st = g->stream;
  // every rank must take the same collective steps: agree on the arguments
  // first (an NCCL group), so that a mismatch fails on every rank alike
  if (g->kind == 1 && g->nranks > 1) {
    DState *s0 = parts[0]->d_st;
    const double mine[6] = {static_cast<double>(solver), static_cast<double>(maxIt),
                            static_cast<double>(newX != 0), -static_cast<double>(solver),
                            -static_cast<double>(maxIt), -static_cast<double>(newX != 0)};
    double agreed[6];
    CK(cudaMemcpyAsync(s0->loc, mine, sizeof(mine), cudaMemcpyHostToDevice, st));
    NK(nccl().AllReduce(s0->loc, s0->glob, 6, ncclDouble, ncclMax, g->comm, st));
    CK(cudaMemcpyAsync(agreed, s0->glob, sizeof(agreed), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int v = 0; v < 3; ++v)
      if (agreed[v] != -agreed[v + 3])
        return fail("the ranks passed different solver, maxIt or newX");
  }
  if (solver != SFR_PCG && solver != SFR_PBICGSTAB)
    return fail("the partitioned path runs PCG and PBICGSTAB", SFR_UNSUPPORTED);
  if (g->kind == 0 && !g->wired) {
    const int rc = wire_local(g);
    if (rc != SFR_OK) return rc;
  }
  const bool pcg = solver == SFR_PCG;
  for (int k = 0; k < nlocal; ++k) {
    sfr_dist *d = parts[k];
    CK(cudaMemcpyAsync(d->b, b[k], d->n * sizeof(double), cudaMemcpyHostToDevice, st));
    if (!newX)
      CK(cudaMemcpyAsync(d->x, x[k], d->ncols * sizeof(double), cudaMemcpyHostToDevice, st));
    DState h{};
    h.active = maxIt > 0 ? 1 : 0;
    h.status = maxIt > 0 ? SFR_OK : SFR_MAXIT;
    h.iters = 1;
    h.maxit = maxIt;
    h.tol = tol;
    CK(cudaMemcpyAsync(d->d_st, &h, sizeof(DState), cudaMemcpyHostToDevice, st));
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int rc = SFR_OK;
  auto launch = [&](auto kernel, auto... extra) -> int {
    for (int k = 0; k < nlocal; ++k)
      kernel<<<wave_grid(kernel, parts[k]), kThreads, 0, st>>>(args_of(parts[k]), extra...);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SFR_OK : cuda_fail(e, "kernel launch");
  };
  auto run = [&]() -> int {
    int r;
    CK(cudaEventRecord(e0, st));
    // setup (Cg.c:283-316, Bicgstab.c:325-346)
    if (pcg) {
      if ((r = launch(k_pcg_setup, newX ? 1 : 0)) != SFR_OK) return r;
    } else {
      if ((r = launch(k_bicg_setup, newX ? 1 : 0)) != SFR_OK) return r;
    }
    if ((r = rank_sum(g, parts, 0, 1, false)) != SFR_OK) return r;
    if (!newX && (r = exchange(g, parts, nlocal, 0, true)) != SFR_OK) return r;
    if (pcg) {
      if ((r = launch(k_pcg_start)) != SFR_OK) return r;
      if ((r = rank_sum(g, parts, 1, 1, false)) != SFR_OK) return r;
    } else if ((r = launch(k_bicg_start)) != SFR_OK) {
      return r;
    }
    // one iteration's launches (Cg.c:322-366, Bicgstab.c:350-437)
    auto iteration = [&]() -> int {
      int q;
      if (pcg) {
        if ((q = exchange(g, parts, nlocal, 1, false)) != SFR_OK) return q;
        if ((q = launch(k_pcg_a)) != SFR_OK) return q;
        if ((q = rank_sum(g, parts, 2, 1, false)) != SFR_OK) return q;
        if ((q = launch(k_pcg_b)) != SFR_OK) return q;
        if ((q = rank_sum(g, parts, 3, 1, false)) != SFR_OK) return q;
        return launch(k_pcg_c);
      }
      if ((q = exchange(g, parts, nlocal, 2, false)) != SFR_OK) return q;
      if ((q = launch(k_bicg_a1)) != SFR_OK) return q;
      if ((q = rank_sum(g, parts, 0, 2, false)) != SFR_OK) return q;
      if ((q = launch(k_bicg_b1)) != SFR_OK) return q;
      if ((q = rank_sum(g, parts, 2, 1, false)) != SFR_OK) return q;
      if ((q = exchange(g, parts, nlocal, 2, false)) != SFR_OK) return q;
      if ((q = launch(k_bicg_a2)) != SFR_OK) return q;
      if ((q = rank_sum(g, parts, 3, 2, false)) != SFR_OK) return q;
      if ((q = launch(k_bicg_b2)) != SFR_OK) return q;
      if ((q = rank_sum(g, parts, 5, 2, false)) != SFR_OK) return q;
      return launch(k_bicg_c);
    };
    // the loop: a graph of kChunk iterations (captured once for this set of
    // ranks), replayed until the ranks agree that the solve stopped; the
    // kernels stop by themselves at maxIt, so a replay past the end is idle
    const int which = pcg ? 0 : 1;
    if (!g->chunk[which] || g->chunk_epoch[which] != g->epoch) {
      if (g->chunk[which]) cudaGraphExecDestroy(g->chunk[which]);
      g->chunk[which] = nullptr;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      int q = SFR_OK;
      for (int it = 0; it < kChunk && q == SFR_OK; ++it) q = iteration();
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(st, &graph);
      if (q != SFR_OK) {
        if (graph) cudaGraphDestroy(graph);
        return q;
      }
      CK(ec);
      const cudaError_t ei = cudaGraphInstantiate(&g->chunk[which], graph, 0);
      cudaGraphDestroy(graph);
      CK(ei);
      g->chunk_epoch[which] = g->epoch;
    }
    DState *s0 = parts[0]->d_st;
    const uint64_t nchunks = (static_cast<uint64_t>(maxIt) + kChunk - 1) / kChunk;
    int prev = -1;
    for (uint64_t c = 0; c < nchunks; ++c) {
      const int slot = static_cast<int>(c & 1);
      CK(cudaGraphLaunch(g->chunk[which], st));
      // the stop flag, agreed over the ranks, read one chunk behind
      if (g->kind == 1 && g->nranks > 1) {
        NK(nccl().AllReduce(&s0->active, &s0->active_all, 1, ncclInt32, ncclMax, g->comm, st));
        CK(cudaMemcpyAsync(g->h_flag + slot, &s0->active_all, sizeof(int),
                           cudaMemcpyDeviceToHost, st));
      } else {
        CK(cudaMemcpyAsync(g->h_flag + slot, &s0->active, sizeof(int), cudaMemcpyDeviceToHost,
                           st));
      }
      CK(cudaEventRecord(g->flag_ev[slot], st));
      if (prev >= 0) {
        CK(cudaEventSynchronize(g->flag_ev[prev]));
        if (g->h_flag[prev] == 0) break;
      }
      prev = slot;
    }
    // post-processing (Cg.c:376-396, Bicgstab.c:440-455)
    if ((r = exchange(g, parts, nlocal, 0, true)) != SFR_OK) return r;
    if ((r = launch(k_post, pcg ? 1 : 0)) != SFR_OK) return r;
    if ((r = rank_sum(g, parts, 0, 5, true)) != SFR_OK) return r;
    CK(cudaEventRecord(e1, st));
    return SFR_OK;
  };
  rc = run();
  if (rc == SFR_OK) {
    DState h;
    CK(cudaMemcpyAsync(&h, parts[0]->d_st, sizeof(DState), cudaMemcpyDeviceToHost, st));
    for (int k = 0; k < nlocal; ++k)
      CK(cudaMemcpyAsync(x[k], parts[k]->x, parts[k]->ncols * sizeof(double),
                         cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (info) {
      std::memset(info, 0, sizeof(*info));
      info->iters = h.iters;
      info->status = h.status;
      info->xKx = h.glob[0];
      info->norm_x = std::sqrt(h.glob[1]);
      info->norm_r_m = pcg ? std::sqrt(std::fabs(h.glob[2])) : NAN;
      info->norm_r = std::sqrt(h.glob[3]);
      info->conv = h.conv;
      info->seconds = ms * 1e-3;
      info->relres = h.glob[4] > 0 ? info->norm_r / std::sqrt(h.glob[4]) : info->norm_r;
    }
    rc = h.status;
  } else {
    cudaStreamSynchronize(st);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int sfr_gpu_dist_destroy(sfr_dist *d) {
  if (!d) return SFR_OK;
  if (d->g) {
    cudaSetDevice(d->device);
    cudaStreamSynchronize(d->g->stream);
    if (d->g->kind == 0) {
      if (d->rank < static_cast<int>(d->g->members.size()) && d->g->members[d->rank] == d)
        d->g->members[d->rank] = nullptr;
      d->g->wired = false;
    } else {
      d->g->members.clear();
    }
    ++d->g->epoch;
  }
  free_dist(d);
  delete d;
  return SFR_OK;
}

}  // extern "C"
