// Autotuner of one system's solve: the engine and the graph engine's launch
// shape, chosen by timing each candidate on the caller's own system.
//
// Candidates (PCG and BiCGSTAB, any K, FP64 or mixed), searched in two
// stages:
//   1. the graph engine at 256 and 128 threads a block, with the SpMV phases
//      as one wave of resident blocks or at 2 or 8 SELL slices (64 or 256
//      rows) per warp; the persistent engine (the whole solve in one
//      cooperative launch); the resident engine, for mixed PCG with one
//      right-hand side when the system fits it;
//      for FP64 PCG with one right-hand side, also the graph engine with the
//      fused iteration (one cooperative kernel an iteration, k_pcg_fused);
//   2. when the graph engine leads with three kernels an iteration: its best
//      shape with the SpMV phases' L2 prefetch 1, 2 or 4 rounds ahead.
// Each candidate solves the caller's right-hand side once untimed (the graph
// is built and the clocks are up), then twice timed with CUDA events; its
// time is the faster of the two.  The automatic choice is kept unless a
// candidate beats it by more than 2 %, so timing noise does not flip the
// choice between two shapes that run alike.  The choice is kept in the
// handle (the automatic engine, 0, then takes it for that kind of solve) and,
// when SFR_TUNE_CACHE names a file, in that file, keyed by the GPU, the
// system's size, pattern and storage and the kind of solve; a later tune of
// the same key reads it back instead of measuring.
//
// The reference has no autotuner: its OpenMP solvers balance rows by
// nonzeros (partitionCsrByNonzeros, Csr.c:1827-1942).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace sfr {

const Tuned *find_tuned(const sfr_system *s, int32_t solver, int32_t k, int32_t precision,
                        bool own_diag) {
  for (const Tuned &t : s->tuned)
    if (t.solver == solver && t.k == k && t.precision == precision &&
        t.own_diag == (own_diag ? 1 : 0))
      return &t;
  return nullptr;
}

namespace {

struct Candidate {
  int engine, threads, spw, pf, fused;
  bool operator==(const Candidate &o) const {
    return engine == o.engine && (engine != 2 || (threads == o.threads && spw == o.spw &&
                                                  pf == o.pf && fused == o.fused));
  }
};

constexpr double kMargin = 0.02;  // a candidate must beat the automatic choice by this
std::mutex g_file_mu;

std::string cache_key(const sfr_system *s, int32_t solver, int32_t k, int32_t precision,
                      bool own_diag) {
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, s->device);
  std::string gpu = prop.name;
  for (char &c : gpu)
    if (c == ' ' || c == '\t') c = '_';
  char buf[512];
  std::snprintf(buf, sizeof(buf),
                "sfr-tune-v3 gpu=%s sms=%d n=%d slots=%lld nsrc=%d storage=%d unsym=%d "
                "off16=%d solver=%d k=%d precision=%d own_diag=%d",
                gpu.c_str(), prop.multiProcessorCount, s->n,
                static_cast<long long>(s->A.nslots), s->nsrc, s->storage, s->unsym,
                s->A.off ? 1 : 0, solver, k, precision, own_diag ? 1 : 0);
  return buf;
}

// The last entry of `key` in the cache file, if any.
bool file_lookup(const std::string &key, Tuned *t) {
  const char *path = std::getenv("SFR_TUNE_CACHE");
  if (!path || !*path) return false;
  std::lock_guard<std::mutex> lk(g_file_mu);
  FILE *f = std::fopen(path, "r");
  if (!f) return false;
  bool found = false;
  std::vector<char> line(4096);
  const std::string head = key + " -> ";
  while (std::fgets(line.data(), static_cast<int>(line.size()), f)) {
    if (std::strncmp(line.data(), head.c_str(), head.size()) != 0) continue;
    int e = 0, th = 0, sp = 0, pf = 0, fu = 0;
    double ms = 0.0;
    if (std::sscanf(line.data() + head.size(),
                    "engine=%d threads=%d spw=%d pf=%d fused=%d ms=%lf", &e, &th, &sp, &pf, &fu,
                    &ms) == 6 &&
        (e == 1 || e == 2 || e == 4) && (th == 128 || th == 256) && sp >= 0 && sp <= 64 &&
        pf >= 0 && pf <= 8 && fu >= 0 && fu <= 4) {
      t->engine = e;
      t->threads = th;
      t->spw = sp;
      t->pf = pf;
      t->fused = fu;
      t->ms = ms;
      found = true;
    }
  }
  std::fclose(f);
  return found;
}

void file_store(const std::string &key, const Tuned &t) {
  const char *path = std::getenv("SFR_TUNE_CACHE");
  if (!path || !*path) return;
  std::lock_guard<std::mutex> lk(g_file_mu);
  FILE *f = std::fopen(path, "a");
  if (!f) return;
  std::fprintf(f, "%s -> engine=%d threads=%d spw=%d pf=%d fused=%d ms=%.6f\n", key.c_str(),
               t.engine, t.threads, t.spw, t.pf, t.fused, t.ms);
  std::fclose(f);
}

void store(sfr_system *s, const Tuned &t) {
  for (Tuned &e : s->tuned)
    if (e.solver == t.solver && e.k == t.k && e.precision == t.precision &&
        e.own_diag == t.own_diag) {
      e = t;
      return;
    }
  s->tuned.push_back(t);
}

void fill(sfr_tune_result *out, const Tuned &t, const Candidate &def, double def_ms, int n,
          int source) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->engine = t.engine;
  out->threads = t.threads;
  out->slices_per_warp = t.spw;
  out->prefetch = t.pf;
  out->fused = t.fused;
  out->ms = t.ms;
  out->default_engine = def.engine;
  out->default_threads = def.threads;
  out->default_slices_per_warp = def.spw;
  out->default_prefetch = def.pf;
  out->default_fused = def.fused;
  out->default_ms = def_ms;
  out->candidates = n;
  out->source = source;
}

}  // namespace
}  // namespace sfr

extern "C" int sfr_gpu_autotune(sfr_system *s, int32_t solver, int32_t k, const double *ad_k,
                                const double *b, double tol, uint32_t maxit, int32_t precision,
                                sfr_tune_result *out) {
  using namespace sfr;
  if (!s || !b || k < 1 || k > 4 || maxit == 0) return SFR_BAD_INPUT;
  if (solver != SFR_PCG && solver != SFR_PBICGSTAB) return SFR_UNSUPPORTED;
  if (precision != SFR_FP64 && precision != SFR_MIXED) return SFR_UNSUPPORTED;
  if (!s->values_set) {
    set_last_error("sfr_gpu_set_values was not called");
    return SFR_BAD_INPUT;
  }
  if (cudaSetDevice(s->device) != cudaSuccess) return SFR_CUDA_ERROR;
  const bool own_diag = ad_k == nullptr;
  const Candidate def{auto_engine(s, solver, k, precision, own_diag), s->graph_threads,
                      s->graph_spw, s->graph_pf, s->graph_fused};
  if (const Tuned *t = find_tuned(s, solver, k, precision, own_diag)) {
    fill(out, *t, def, 0.0, 0, 1);
    return SFR_OK;
  }
  const std::string key = cache_key(s, solver, k, precision, own_diag);
  Tuned t;
  t.solver = solver;
  t.k = k;
  t.precision = precision;
  t.own_diag = own_diag ? 1 : 0;
  if (file_lookup(key, &t)) {
    store(s, t);
    fill(out, t, def, 0.0, 0, 2);
    return SFR_OK;
  }

  std::vector<Candidate> cands{def};
  auto add = [&](const Candidate &c) {
    if (std::find(cands.begin(), cands.end(), c) == cands.end()) cands.push_back(c);
  };
  for (int th : {256, 128})
    for (int sp : {0, 2, 8}) add({2, th, sp, 0, 0});
  if (precision == SFR_FP64 && solver == SFR_PCG && k == 1) {
    for (int mode : {1, 2, 3, 4}) add({2, 256, 0, 0, mode});
  }
  add({1, 0, 0, 0, 0});
  if (precision == SFR_MIXED && solver == SFR_PCG && k == 1 && own_diag && resident_fits(s))
    add({4, 0, 0, 0, 0});

  // device copies of the right-hand sides (and diagonals); a scratch x
  const size_t total = static_cast<size_t>(s->n) * k;
  double *d_b = nullptr, *d_x = nullptr, *d_ad = nullptr;
  auto release = [&] {
    cudaFree(d_b);
    cudaFree(d_x);
    cudaFree(d_ad);
  };
  if (cudaMalloc(&d_b, sizeof(double) * total) != cudaSuccess ||
      cudaMalloc(&d_x, sizeof(double) * total) != cudaSuccess ||
      (ad_k && cudaMalloc(&d_ad, sizeof(double) * total) != cudaSuccess) ||
      cudaMemcpy(d_b, b, sizeof(double) * total, cudaMemcpyHostToDevice) != cudaSuccess ||
      (ad_k && cudaMemcpy(d_ad, ad_k, sizeof(double) * total, cudaMemcpyHostToDevice) !=
                   cudaSuccess)) {
    release();
    return SFR_CUDA_ERROR;
  }
  const int32_t engine0 = s->engine, threads0 = s->graph_threads, spw0 = s->graph_spw;
  std::vector<double> ms(cands.size(), std::numeric_limits<double>::infinity());
  std::vector<sfr_solve_info> info(k);
  int hard = SFR_OK;
  int timed = 0;
  const int32_t pf0 = s->graph_pf, fused0 = s->graph_fused;
  // time candidates [from, cands.size())
  auto measure = [&](size_t from) {
    ms.resize(cands.size(), std::numeric_limits<double>::infinity());
    for (size_t c = from; c < cands.size() && hard == SFR_OK; ++c) {
      s->engine = cands[c].engine;
      s->graph_threads = cands[c].threads ? cands[c].threads : threads0;
      s->graph_spw = cands[c].spw;
      s->graph_pf = cands[c].pf;
      s->graph_fused = cands[c].fused;
      double best = std::numeric_limits<double>::infinity();
      bool ok = true;
      for (int rep = 0; rep < 3 && ok; ++rep) {
        const int rc = solve_device(s, solver, k, d_ad, d_b, d_x, tol, maxit, 1, precision,
                                    s->stream, info.data());
        if (rc == SFR_CUDA_ERROR || rc == SFR_TIMEOUT) {
          hard = rc;
          ok = false;
        } else if (rc != SFR_OK) {
          ok = false;  // this candidate does not serve the solve (unsupported, no convergence)
        } else if (rep > 0) {
          best = std::min(best, info[0].seconds * 1e3);
        }
      }
      if (ok) {
        ms[c] = best;
        ++timed;
      }
    }
  };
  measure(0);
  // stage 2: the L2 prefetch distance on the best graph shape of stage 1
  const size_t stage1 = cands.size();
  size_t lead = 0;
  for (size_t j = 1; j < stage1; ++j)
    if (ms[j] < ms[lead]) lead = j;
  if (hard == SFR_OK && cands[lead].engine == 2 && !cands[lead].fused) {
    for (int pf : {1, 2, 4}) add({2, cands[lead].threads, cands[lead].spw, pf, 0});
    measure(stage1);
  }
  s->engine = engine0;
  s->graph_pf = pf0;
  s->graph_fused = fused0;
  s->graph_threads = threads0;
  s->graph_spw = spw0;
  release();
  if (hard != SFR_OK) return hard;
  if (!(ms[0] < std::numeric_limits<double>::infinity())) {
    set_last_error("sfr_gpu_autotune: the automatic choice does not solve this system");
    return SFR_MAXIT;
  }
  size_t pick = 0;
  for (size_t c = 1; c < cands.size(); ++c)
    if (ms[c] < ms[pick]) pick = c;
  if (pick != 0 && ms[pick] > (1.0 - kMargin) * ms[0]) pick = 0;
  t.engine = cands[pick].engine;
  t.threads = cands[pick].threads ? cands[pick].threads : threads0;
  t.spw = cands[pick].spw;
  t.pf = cands[pick].pf;
  t.fused = cands[pick].fused;
  t.ms = ms[pick];
  store(s, t);
  file_store(key, t);
  fill(out, t, def, ms[0], timed, 0);
  return SFR_OK;
}

extern "C" int sfr_gpu_autotune_clear(sfr_system *s) {
  if (!s) return SFR_BAD_INPUT;
  s->tuned.clear();
  return SFR_OK;
}
