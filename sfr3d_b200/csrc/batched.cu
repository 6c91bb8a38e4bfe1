// Batched solves: many independent systems of uneven size in one persistent
// cooperative launch, replayed from a CUDA graph.
//
// The systems are concatenated into one block-diagonal SELL-32 matrix, each
// system's rows padded to whole slices so that no slice straddles two
// systems.  Each system gets a team of blocks (persist.cuh): its own slice
// range, reductions over its own blocks and its own bounded barrier, so every
// system iterates at its own pace and stops at its own convergence inside the
// single launch.  Blocks are shared out in proportion to each system's work
// per solve (slices x iterations), which the autotuner measures.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "persist.cuh"

struct sfr_batch {
  int32_t device = 0;
  int32_t nsys = 0;
  int32_t storage = 0;
  int32_t unsym = 0;
  std::vector<int32_t> n, row_off, slice_off, nslices, src_off, nsrc;
  sfr_system cat;               // the block-diagonal concatenation
  std::vector<double> weight;   // work per solve: slices x iterations
  std::vector<int> team_blocks; // blocks per team chosen by the autotuner (empty: by weight)
  std::vector<int> blocks_of;   // blocks per team of the installed plan
  std::vector<double> team_ms;  // each team's time in the last solve (ms)
  sfr_batch_tune tune{};        // the last autotune's report
  // launch plan
  int32_t plan_solver = -1, plan_precision = -1, grid = 0;
  sfr::TeamTable table{};
  int4 *d_block = nullptr;
  int2 *d_sys = nullptr;
  unsigned *d_bar = nullptr;
  void *ws = nullptr;
  size_t ws_bytes = 0;
  sfr::SolveOut *d_out = nullptr;
  unsigned *d_ctl = nullptr;
  double *d_b = nullptr, *d_x = nullptr;
  // the captured launch and the scalars baked into it
  cudaGraphExec_t exec = nullptr;
  double g_tol = -1.0;
  uint32_t g_maxit = 0;
  int32_t g_newx = -1;
};

namespace sfr {
namespace {

// Blocks per team from the work weights: in proportion, at least one and at
// most one block per slice of the system, all fitting in `gmax`.
std::vector<int> share_by_weight(const sfr_batch *b, int gmax) {
  const int S = b->nsys;
  double wsum = 0.0;
  for (double w : b->weight) wsum += w;
  std::vector<int> nb(S);
  std::vector<double> raw(S);
  int total = 0;
  for (int s = 0; s < S; ++s) {
    raw[s] = gmax * b->weight[s] / wsum;
    nb[s] = std::max(1, std::min(static_cast<int>(raw[s]), b->nslices[s]));
    total += nb[s];
  }
  while (total > gmax) {  // trim the largest teams
    int big = 0;
    for (int s = 1; s < S; ++s)
      if (nb[s] > nb[big]) big = s;
    if (nb[big] <= 1) break;
    --nb[big];
    --total;
  }
  while (total < gmax) {  // hand leftovers to the most under-served teams
    int best = -1;
    double deficit = 0.0;
    for (int s = 0; s < S; ++s) {
      if (nb[s] >= b->nslices[s]) continue;
      const double d = raw[s] - nb[s];
      if (best < 0 || d > deficit) {
        best = s;
        deficit = d;
      }
    }
    if (best < 0 || deficit <= 0.0) break;
    ++nb[best];
    ++total;
  }
  return nb;
}

int max_grid(const sfr_batch *b, int32_t solver, int32_t precision) {
  return precision == SFR_MIXED ? team_max_grid_mixed(solver, b->device)
                                : team_max_grid_fp64(solver, b->device);
}

// Install a launch plan: team s gets nb[s] blocks (b->team_blocks when set
// by the autotuner, else shares of the work weights).
int plan(sfr_batch *b, int32_t solver, int32_t precision) {
  const int gmax = max_grid(b, solver, precision);
  if (gmax <= 0) return SFR_CUDA_ERROR;
  if (b->nsys > gmax) {
    set_last_error("more systems than co-resident blocks in one launch");
    return SFR_UNSUPPORTED;
  }
  const int S = b->nsys;
  std::vector<int> nb;
  int total = 0;
  if (static_cast<int>(b->team_blocks.size()) == S) {
    nb = b->team_blocks;
    for (int s = 0; s < S; ++s) {
      nb[s] = std::max(1, std::min(nb[s], b->nslices[s]));
      total += nb[s];
    }
    if (total > gmax) nb = share_by_weight(b, gmax);
  } else {
    nb = share_by_weight(b, gmax);
  }
  total = 0;
  for (int v : nb) total += v;
  b->blocks_of = nb;
  std::vector<int4> blocks;
  std::vector<int2> sys;
  blocks.reserve(total);
  sys.reserve(total);
  for (int s = 0; s < S; ++s) {
    const int b0 = static_cast<int>(blocks.size());
    const int64_t ns = b->nslices[s];
    for (int j = 0; j < nb[s]; ++j) {
      const int s0 = b->slice_off[s] + static_cast<int>(ns * j / nb[s]);
      const int s1 = b->slice_off[s] + static_cast<int>(ns * (j + 1) / nb[s]);
      blocks.push_back(make_int4(s0, s1, b0, b0 + nb[s]));
      sys.push_back(make_int2(s, b->row_off[s] + b->n[s]));
    }
  }
  const int grid = static_cast<int>(blocks.size());
  cudaFree(b->d_block);
  cudaFree(b->d_sys);
  b->d_block = nullptr;
  b->d_sys = nullptr;
  if (cudaMalloc(&b->d_block, sizeof(int4) * grid) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaMalloc(&b->d_sys, sizeof(int2) * grid) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaMemcpy(b->d_block, blocks.data(), sizeof(int4) * grid, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(b->d_sys, sys.data(), sizeof(int2) * grid, cudaMemcpyHostToDevice) != cudaSuccess)
    return SFR_CUDA_ERROR;
  const size_t need = precision == SFR_MIXED ? team_ws_bytes_mixed(b->cat.n, grid)
                                             : team_ws_bytes_fp64(b->cat.n, grid);
  if (need > b->ws_bytes) {
    cudaFree(b->ws);
    b->ws = nullptr;
    if (cudaMalloc(&b->ws, need) != cudaSuccess) return SFR_CUDA_ERROR;
    b->ws_bytes = need;
  }
  b->grid = grid;
  b->table.block = b->d_block;
  b->table.sys = b->d_sys;
  b->table.bar = b->d_bar;
  b->plan_solver = solver;
  b->plan_precision = precision;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  return SFR_OK;
}

// Capture [clear the team barriers -> one cooperative launch] as a graph.
int capture(sfr_batch *b, int32_t solver, int32_t precision, double tol, uint32_t maxit,
            int32_t newx) {
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return SFR_CUDA_ERROR;
  cudaGraph_t g = nullptr;
  int rc = SFR_OK;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaStreamDestroy(cs);
    return SFR_CUDA_ERROR;
  }
  if (cudaMemsetAsync(b->d_bar, 0, sizeof(unsigned) * 2 * b->nsys, cs) != cudaSuccess)
    rc = SFR_CUDA_ERROR;
  if (rc == SFR_OK)
    rc = precision == SFR_MIXED
             ? enqueue_team_mixed(&b->cat, solver, b->d_b, b->d_x, tol, maxit, newx, b->table,
                                  b->grid, b->ws, b->d_out, b->d_ctl, cs)
             : enqueue_team_fp64(&b->cat, solver, b->d_b, b->d_x, tol, maxit, newx, b->table,
                                 b->grid, b->ws, b->d_out, b->d_ctl, cs);
  const cudaError_t ee = cudaStreamEndCapture(cs, &g);
  if (rc == SFR_OK && ee != cudaSuccess) rc = SFR_CUDA_ERROR;
  if (rc == SFR_OK && cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) rc = SFR_CUDA_ERROR;
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  if (rc == SFR_OK) {
    b->g_tol = tol;
    b->g_maxit = maxit;
    b->g_newx = newx;
  }
  return rc;
}

int run(sfr_batch *b, int32_t solver, double tol, uint32_t maxit, int32_t newx,
        int32_t precision, std::vector<SolveOut> *out, float *ms) {
  int rc;
  if (b->plan_solver != solver || b->plan_precision != precision || !b->d_block) {
    rc = plan(b, solver, precision);
    if (rc != SFR_OK) return rc;
  }
  if (!b->exec || b->g_tol != tol || b->g_maxit != maxit || b->g_newx != newx) {
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    rc = capture(b, solver, precision, tol, maxit, newx);
    if (rc != SFR_OK) return rc;
  }
  cudaStream_t st = b->cat.stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  cudaError_t err = cudaGraphLaunch(b->exec, st);
  cudaEventRecord(e1, st);
  out->resize(b->nsys);
  unsigned ctl[3] = {0, 0, 0};
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(out->data(), b->d_out, sizeof(SolveOut) * b->nsys,
                          cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(ctl, b->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) {
    set_last_error(cudaGetErrorString(err));
    return SFR_CUDA_ERROR;
  }
  if (ctl[2] != 0) return static_cast<int>(ctl[2]);
  return SFR_OK;
}

}  // namespace
}  // namespace sfr

extern "C" {

int sfr_gpu_batch_create(int32_t nsys, const int32_t *neq, const int32_t *nad,
                         const int32_t *const *ia, const int32_t *const *ja, int32_t storage,
                         int32_t unsym, int32_t device, sfr_batch **out) {
  if (!out || nsys <= 0 || !neq || !ia) return SFR_BAD_INPUT;
  *out = nullptr;
  auto b = std::make_unique<sfr_batch>();
  b->device = device;
  b->nsys = nsys;
  b->storage = storage;
  b->unsym = unsym;
  sfr::HostSell cat;
  cat.sptr.push_back(0);
  int64_t rows = 0, slices = 0, src = 0;
  for (int s = 0; s < nsys; ++s) {
    sfr::HostSell h;
    std::string why;
    int32_t ns = 0;
    const int rc = sfr::build_sell(neq[s], nad ? nad[s] : 0, ia[s], ja ? ja[s] : nullptr,
                                   storage, unsym, &h, nullptr, &ns, &why);
    if (rc != SFR_OK) {
      sfr::set_last_error(("system " + std::to_string(s) + ": " + why).c_str());
      return rc;
    }
    b->n.push_back(neq[s]);
    b->row_off.push_back(static_cast<int32_t>(rows));
    b->slice_off.push_back(static_cast<int32_t>(slices));
    b->nslices.push_back(h.nslices);
    b->src_off.push_back(static_cast<int32_t>(src));
    b->nsrc.push_back(ns);
    const int32_t slot0 = cat.sptr.back();
    for (int32_t k = 1; k <= h.nslices; ++k) cat.sptr.push_back(slot0 + h.sptr[k]);
    for (size_t e = 0; e < h.col.size(); ++e) {
      cat.col.push_back(h.col[e] + static_cast<int32_t>(rows));
      cat.src.push_back(h.src[e] >= 0 ? h.src[e] + static_cast<int32_t>(src) : -1);
    }
    rows += static_cast<int64_t>(h.nslices) * sfr::kWarpHost;
    slices += h.nslices;
    src += ns;
    if (rows > INT32_MAX || src > INT32_MAX || cat.sptr.back() < 0) return SFR_BAD_INPUT;
    // default work estimate: slices x an iteration count growing like n^(1/3)
    b->weight.push_back(static_cast<double>(h.nslices) * std::cbrt(static_cast<double>(neq[s])));
  }
  b->team_ms.assign(nsys, 0.0);
  cat.n = static_cast<int32_t>(rows);
  cat.nslices = static_cast<int32_t>(slices);
  sfr_system &c = b->cat;
  c.device = device;
  c.n = cat.n;
  c.storage = storage;
  c.unsym = unsym;
  c.nsrc = static_cast<int32_t>(src);
  if (cudaSetDevice(device) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess)
    return SFR_CUDA_ERROR;
  int rc = sfr::upload_sell(cat, &c.A, &c.bytes);
  if (rc != SFR_OK) return rc;
  const size_t nrow = static_cast<size_t>(c.n);
  if (cudaMalloc(&c.d_stage, sizeof(double) * std::max<int64_t>(src, 1)) != cudaSuccess ||
      cudaMalloc(&c.d_diag, sizeof(double) * nrow) != cudaSuccess ||
      cudaMalloc(&c.d_diag32, sizeof(float) * nrow) != cudaSuccess ||
      cudaMalloc(&b->d_b, sizeof(double) * nrow) != cudaSuccess ||
      cudaMalloc(&b->d_x, sizeof(double) * nrow) != cudaSuccess ||
      cudaMalloc(&b->d_bar, sizeof(unsigned) * 2 * nsys) != cudaSuccess ||
      cudaMalloc(&b->d_out, sizeof(sfr::SolveOut) * nsys) != cudaSuccess ||
      cudaMalloc(&b->d_ctl, 64) != cudaSuccess)
    return SFR_CUDA_ERROR;
  // padding rows: unit diagonal, zero right-hand side and solution
  std::vector<double> ones(nrow, 1.0);
  if (cudaMemcpy(c.d_diag, ones.data(), sizeof(double) * nrow, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemset(b->d_b, 0, sizeof(double) * nrow) != cudaSuccess ||
      cudaMemset(b->d_x, 0, sizeof(double) * nrow) != cudaSuccess)
    return SFR_CUDA_ERROR;
  *out = b.release();
  return SFR_OK;
}

int sfr_gpu_batch_set_values(sfr_batch *b, const double *const *al, const double *const *ad,
                             const double *const *au) {
  if (!b || !ad || !al) return SFR_BAD_INPUT;
  sfr_system &c = b->cat;
  if (cudaSetDevice(b->device) != cudaSuccess) return SFR_CUDA_ERROR;
  const bool split = b->storage == SFR_CSRC && b->unsym;
  for (int s = 0; s < b->nsys; ++s) {
    if (!ad[s] || (!al[s] && b->nsrc[s] > 0)) return SFR_BAD_INPUT;
    double *dst = c.d_stage + b->src_off[s];
    if (split && au && au[s]) {
      const size_t half = static_cast<size_t>(b->nsrc[s]) / 2;
      if (cudaMemcpyAsync(dst, al[s], sizeof(double) * half, cudaMemcpyHostToDevice, c.stream) !=
              cudaSuccess ||
          cudaMemcpyAsync(dst + half, au[s], sizeof(double) * half, cudaMemcpyHostToDevice,
                          c.stream) != cudaSuccess)
        return SFR_CUDA_ERROR;
    } else if (b->nsrc[s] > 0) {
      if (cudaMemcpyAsync(dst, al[s], sizeof(double) * b->nsrc[s], cudaMemcpyHostToDevice,
                          c.stream) != cudaSuccess)
        return SFR_CUDA_ERROR;
    }
    if (cudaMemcpyAsync(c.d_diag + b->row_off[s], ad[s], sizeof(double) * b->n[s],
                        cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
      return SFR_CUDA_ERROR;
  }
  int rc = sfr::gather_values(&c, &c.A, c.stream);
  if (rc != SFR_OK) return rc;
  rc = sfr::row_compensation(&c, c.A, c.stream);
  if (rc != SFR_OK) return rc;
  if (sfr::convert_diag32(c.d_diag, c.d_diag32, c.n, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess)
    return SFR_CUDA_ERROR;
  c.values_set = true;
  return SFR_OK;
}

int sfr_gpu_batch_solve(sfr_batch *b, int32_t solver, const double *const *bv, double *const *x,
                        double tol, uint32_t maxit, int32_t newx, int32_t precision,
                        sfr_solve_info *info) {
  if (!b || !bv || !x) return SFR_BAD_INPUT;
  if (solver != SFR_PCG && solver != SFR_PBICGSTAB) return SFR_UNSUPPORTED;
  if (precision != SFR_FP64 && precision != SFR_MIXED) return SFR_UNSUPPORTED;
  if (!b->cat.values_set) return SFR_BAD_INPUT;
  if (maxit == 0) return SFR_BAD_INPUT;
  sfr_system &c = b->cat;
  if (cudaSetDevice(b->device) != cudaSuccess) return SFR_CUDA_ERROR;
  for (int s = 0; s < b->nsys; ++s) {
    if (!bv[s] || !x[s]) return SFR_BAD_INPUT;
    const size_t bytes = sizeof(double) * b->n[s];
    if (cudaMemcpyAsync(b->d_b + b->row_off[s], bv[s], bytes, cudaMemcpyHostToDevice, c.stream) !=
        cudaSuccess)
      return SFR_CUDA_ERROR;
    if (!newx && cudaMemcpyAsync(b->d_x + b->row_off[s], x[s], bytes, cudaMemcpyHostToDevice,
                                 c.stream) != cudaSuccess)
      return SFR_CUDA_ERROR;
  }
  std::vector<sfr::SolveOut> out;
  float ms = 0.f;
  int rc = sfr::run(b, solver, tol, maxit, newx, precision, &out, &ms);
  if (rc != SFR_OK) return rc;
  int worst = SFR_OK;
  for (int s = 0; s < b->nsys; ++s) {
    if (cudaMemcpyAsync(x[s], b->d_x + b->row_off[s], sizeof(double) * b->n[s],
                        cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
      return SFR_CUDA_ERROR;
    if (info) {
      sfr_solve_info &f = info[s];
      std::memset(&f, 0, sizeof(f));
      f.iters = out[s].iters;
      f.status = out[s].status;
      f.xKx = out[s].xKx;
      f.norm_x = out[s].norm_x;
      f.norm_r = out[s].norm_r;
      f.norm_r_m = out[s].norm_r_m;
      f.conv = out[s].conv;
      f.seconds = ms * 1e-3;
      f.refinements = out[s].refinements;
      f.inner_iters = out[s].inner_iters;
      f.relres = out[s].bnorm > 0 ? out[s].norm_r / out[s].bnorm : std::nan("");
    }
    b->team_ms[s] = out[s].team_ms;
    if (out[s].status != SFR_OK && worst == SFR_OK) worst = out[s].status;
  }
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return SFR_CUDA_ERROR;
  return worst;
}

int sfr_gpu_batch_set_weights(sfr_batch *b, const double *w) {
  if (!b || !w) return SFR_BAD_INPUT;
  for (int s = 0; s < b->nsys; ++s)
    if (!(w[s] > 0.0)) return SFR_BAD_INPUT;
  b->weight.assign(w, w + b->nsys);
  b->team_blocks.clear();
  b->plan_solver = -1;  // re-plan on the next solve
  return SFR_OK;
}

// Autotuner: the batch's time is its slowest team's, so the blocks are
// shared out to equalise the teams' measured times.
//   1. Measure the default plan (blocks by slices x n^(1/3)) and the plan
//      weighted by slices x measured iterations; every team reports its own
//      time inside the launch (team_ms).
//   2. Fit each team's time to t(B) = f + w / B over the plans measured (f:
//      the barrier- and latency-bound part that more blocks do not shrink,
//      w / B: the part they share).
//   3. Bisect on the target time T for the smallest T whose block counts
//      B_s(T) = ceil(w_s / (T - f_s)) fit in one co-resident launch; hand
//      leftover blocks to the teams predicted slowest.
//   4. Measure that plan, refit, repeat (three model rounds at most); keep
//      the fastest plan measured.  Each plan is timed as the second of two
//      solves (CUDA events), so graph capture is not in the time.
int sfr_gpu_batch_autotune(sfr_batch *b, int32_t solver, const double *const *bv, double tol,
                           uint32_t maxit, int32_t precision, double *ms_out) {
  if (!b || !bv) return SFR_BAD_INPUT;
  const int S = b->nsys;
  std::vector<std::vector<double>> xs(S);
  std::vector<double *> xp(S);
  for (int s = 0; s < S; ++s) {
    xs[s].assign(b->n[s], 0.0);
    xp[s] = xs[s].data();
  }
  const int gmax = sfr::max_grid(b, solver, precision);
  if (gmax <= 0) return SFR_CUDA_ERROR;
  struct Sample {
    std::vector<int> nb;
    std::vector<double> t;
    double total;
  };
  std::vector<Sample> samples;
  std::vector<sfr_solve_info> info(S);
  std::vector<int> iters(S, 1);
  // one plan: install, solve twice, record the second solve's times
  auto measure = [&](const std::vector<int> *nb) -> int {
    if (nb) b->team_blocks = *nb;
    else b->team_blocks.clear();
    b->plan_solver = -1;
    for (int rep = 0; rep < 2; ++rep) {
      const int rc = sfr_gpu_batch_solve(b, solver, bv, xp.data(), tol, maxit, 1, precision,
                                         info.data());
      if (rc < 0) return rc;
    }
    Sample smp;
    smp.nb = b->blocks_of;
    smp.total = info[0].seconds * 1e3;
    smp.t.resize(S);
    for (int s = 0; s < S; ++s) {
      smp.t[s] = b->team_ms[s];
      iters[s] = std::max(1, info[s].inner_iters > 0 ? info[s].inner_iters : info[s].iters);
    }
    samples.push_back(std::move(smp));
    return SFR_OK;
  };
  const std::vector<double> w_default = b->weight;
  int rc = measure(nullptr);  // the default work estimate
  if (rc != SFR_OK) return rc;
  std::vector<double> w1(S);
  for (int s = 0; s < S; ++s) w1[s] = static_cast<double>(b->nslices[s]) * iters[s];
  b->weight = w1;
  rc = measure(nullptr);  // weighted by measured iterations
  if (rc != SFR_OK) return rc;

  for (int round = 0; round < 3; ++round) {
    // fit t = f + w / B per team (least squares over the distinct B seen)
    std::vector<double> f(S), w(S);
    for (int s = 0; s < S; ++s) {
      double su = 0, sv = 0, suu = 0, suv = 0;
      int m = 0;
      for (const Sample &smp : samples) {
        const double u = 1.0 / smp.nb[s];
        su += u;
        sv += smp.t[s];
        suu += u * u;
        suv += u * smp.t[s];
        ++m;
      }
      const double den = m * suu - su * su;
      double ws = 0.0, fs = 0.0;
      if (m >= 2 && den > 1e-18 * m * suu) {
        ws = (m * suv - su * sv) / den;
        fs = (sv - ws * su) / m;
      }
      if (!(ws > 0.0) || !(fs >= 0.0)) {
        // one block count seen, or times that do not shrink with more
        // blocks: split the latest time evenly into the two parts
        const Sample &last = samples.back();
        fs = 0.5 * last.t[s];
        ws = 0.5 * last.t[s] * last.nb[s];
      }
      f[s] = fs;
      w[s] = ws;
    }
    auto need = [&](int s, double T) -> int {  // blocks team s needs for time T
      if (T <= f[s]) return INT32_MAX;
      const double bl = std::ceil(w[s] / (T - f[s]) - 1e-9);
      return bl > INT32_MAX / 2 ? INT32_MAX : std::max(1, static_cast<int>(bl));
    };
    auto fits = [&](double T) {
      int64_t tot = 0;
      for (int s = 0; s < S; ++s) {
        const int bl = need(s, T);
        if (bl > b->nslices[s]) return false;
        tot += bl;
      }
      return tot <= gmax;
    };
    double hi = 0.0;
    for (int s = 0; s < S; ++s) hi = std::max(hi, f[s] + w[s]);  // one block each
    double lo = 0.0;
    if (!fits(hi)) break;  // the model cannot place every team
    for (int it = 0; it < 60; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (fits(mid)) hi = mid;
      else lo = mid;
    }
    std::vector<int> nb(S);
    int total = 0;
    for (int s = 0; s < S; ++s) {
      nb[s] = need(s, hi);
      total += nb[s];
    }
    while (total < gmax) {  // leftovers to the teams predicted slowest
      int worst = -1;
      double tw = -1.0;
      for (int s = 0; s < S; ++s) {
        if (nb[s] >= b->nslices[s]) continue;
        const double t = f[s] + w[s] / nb[s];
        if (t > tw) {
          tw = t;
          worst = s;
        }
      }
      if (worst < 0) break;
      ++nb[worst];
      ++total;
    }
    bool seen = false;
    for (const Sample &smp : samples) seen = seen || smp.nb == nb;
    if (seen) break;  // converged on a plan already measured
    rc = measure(&nb);
    if (rc != SFR_OK) return rc;
  }
  size_t best = 0;
  for (size_t i = 1; i < samples.size(); ++i)
    if (samples[i].total < samples[best].total) best = i;
  // keep the best plan
  if (best == 0) {
    b->weight = w_default;
    b->team_blocks.clear();
  } else if (best == 1) {
    b->team_blocks.clear();
  } else {
    b->team_blocks = samples[best].nb;
  }
  b->plan_solver = -1;
  sfr_batch_tune &r = b->tune;
  r.default_ms = samples[0].total;
  r.weighted_ms = samples[1].total;
  r.tuned_ms = samples[best].total;
  r.plans = static_cast<int32_t>(samples.size());
  r.kept = static_cast<int32_t>(best);
  int g = 0, mx = 0, mn = INT32_MAX;
  for (int v : samples[best].nb) {
    g += v;
    mx = std::max(mx, v);
    mn = std::min(mn, v);
  }
  r.grid = g;
  r.max_team_blocks = mx;
  r.min_team_blocks = mn;
  if (ms_out) *ms_out = samples[best].total;
  return SFR_OK;
}

int sfr_gpu_batch_tune_report(const sfr_batch *b, sfr_batch_tune *out) {
  if (!b || !out) return SFR_BAD_INPUT;
  *out = b->tune;
  return SFR_OK;
}

int sfr_gpu_batch_stats(const sfr_batch *b, int32_t *grid, int64_t *rows, int64_t *bytes) {
  if (!b) return SFR_BAD_INPUT;
  if (grid) *grid = b->grid;
  if (rows) *rows = b->cat.n;
  if (bytes) *bytes = b->cat.bytes + static_cast<int64_t>(b->ws_bytes);
  return SFR_OK;
}

int sfr_gpu_batch_destroy(sfr_batch *b) {
  if (!b) return SFR_OK;
  cudaSetDevice(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  sfr::free_sell(&b->cat.A);
  cudaFree(b->cat.d_stage);
  cudaFree(b->cat.d_diag);
  cudaFree(b->cat.d_diag32);
  cudaFree(b->cat.d_comp);
  if (b->cat.stream) cudaStreamDestroy(b->cat.stream);
  cudaFree(b->d_block);
  cudaFree(b->d_sys);
  cudaFree(b->d_bar);
  cudaFree(b->ws);
  cudaFree(b->d_out);
  cudaFree(b->d_ctl);
  cudaFree(b->d_b);
  cudaFree(b->d_x);
  delete b;
  return SFR_OK;
}

}  // extern "C"
