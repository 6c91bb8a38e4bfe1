// Internal host-side structures of libsfr3d_b200.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "sfr3d_b200.h"

namespace sfr {

constexpr int kWarpHost = 32;  // rows per SELL slice (one warp)

// SELL-32 layout built on the host from one of the reference's layouts.
// src[e] is the index of slot e's value in the value source the caller
// passes (al, or al|au for CSRC unsym), or -1 for a padded slot.
struct HostSell {
  int32_t n = 0;
  int32_t nslices = 0;
  std::vector<int32_t> sptr;  // nslices + 1, in slots
  std::vector<int32_t> col;
  std::vector<int32_t> src;
  int32_t bandwidth = 0;
  int32_t max_width = 0;
  int64_t nnz = 0;  // real (non-padded) off-diagonal slots
};

// Validates the reference layout and builds the SELL copy of A (and, when
// `transpose` is set, of A^T).  Returns SFR_OK or SFR_BAD_INPUT with a
// message in *why.
int build_sell(int32_t neq, int32_t nad, const int32_t *ia, const int32_t *ja,
               int32_t storage, int32_t unsym, HostSell *a, HostSell *at,
               int32_t *nsrc, std::string *why);

// Device copy of one SELL matrix.
struct DevSell {
  int32_t n = 0, nslices = 0;
  int64_t nslots = 0;
  int32_t *sptr = nullptr, *col = nullptr, *src = nullptr;
  int16_t *off = nullptr;  // col - row per slot (0 in padding rows); null when the
                           // bandwidth exceeds 32767
  double *val = nullptr;  // FP64 values
  float *val32 = nullptr; // FP32 copy (mixed precision)
  int32_t max_width = 0;  // slots of the widest slice
};

struct SolveOut;  // device-side result record (krylov.cu)

// An autotuned engine and launch shape for one kind of solve of a system
// (autotune.cpp); the automatic engine choice (engine 0) takes it.
struct Tuned {
  int32_t solver = 0, k = 0, precision = 0, own_diag = 0;  // the kind of solve
  int32_t engine = 0, threads = 0, spw = 0, pf = 0, fused = 0;  // the choice
  double ms = 0.0;
};

struct Workspace {
  size_t bytes = 0;
  void *base = nullptr;
};

}  // namespace sfr

struct sfr_system {
  int32_t device = 0;
  int32_t n = 0;
  int32_t storage = 0;
  int32_t unsym = 0;
  int32_t nad = 0;
  int32_t nsrc = 0;  // length of the value source (al[, au])
  int32_t bandwidth = 0;
  sfr::HostSell host_at;    // kept until A^T is first needed
  bool have_at_host = false;
  sfr::DevSell A, At;
  bool at_ready = false;
  double *d_stage = nullptr;   // raw al|au
  double *d_diag = nullptr;    // ad
  // -sum over each row of (fl32(a_ij) - a_ij): added to the diagonal of the
  // FP32 operator so that it keeps the FP64 row sums (mixed precision)
  double *d_comp = nullptr;
  float *d_diag32 = nullptr;
  bool values_set = false;
  cudaStream_t stream = nullptr;
  sfr::Workspace ws;
  // the transposed view used by the adjoint (shares A^T, diagonal, values)
  sfr_system *tview = nullptr;
  bool borrowed = false;     // a view: its matrix buffers belong to another handle
  bool comp_stale = true;    // compensation not yet computed for the current values
  // resident engine (resident.cu): the symmetrically scaled FP32 operator,
  // rebuilt when the values or the diagonal change
  float *d_rval = nullptr;      // fl32(a_ij / sqrt(ad_i ad_j)) per SELL slot
  float *d_rdelta = nullptr;    // per row: correction of the unit diagonal
  int *d_rbad = nullptr;        // set when a diagonal entry is not positive
  uint64_t values_epoch = 0;    // bumped by every value / diagonal upload
  uint64_t resident_epoch = ~0ull;  // epoch the scaled operator was built for
  bool resident_ok = false;     // the diagonal was positive at that epoch
  // engine: 0 auto, 1 persistent (one cooperative launch), 2 graph,
  // 3 the graph engine's kernels from a host loop (profiling),
  // 4 resident (mixed PCG with the inner iteration on chip)
  int32_t engine = 0;
  int32_t graph_threads = 256;   // graph engine launch shape
  int32_t graph_spw = 0;         // SELL slices per warp; 0: one wave of resident blocks
  int32_t graph_pf = 0;          // SpMV-phase L2 prefetch distance (rounds); 0: off
  int32_t graph_fused = 4;       // FP64 PCG, one RHS: the fused iteration's mode (4: one launch a solve)
  int32_t graph_stage = 0;       // BiCGSTAB SpMV phases: slices staged in shared memory
  std::vector<sfr::Tuned> tuned; // autotuned choices, used when engine == 0
  int64_t bytes = 0;
};

namespace sfr {
int upload_sell(const HostSell &h, DevSell *d, int64_t *bytes);
void free_sell(DevSell *d);
int ensure_workspace(sfr_system *s, size_t bytes);
int gather_values(sfr_system *s, DevSell *d, cudaStream_t st);
// the derived copies and epoch after new raw values and diagonal (capi.cpp)
int values_refreshed(sfr_system *s, cudaStream_t st, bool a_done = false);
cudaError_t convert_diag32(const double *src, float *dst, int n, cudaStream_t st);
// d_comp from the FP64 and FP32 values of d (allocates d_comp on first use)
int row_compensation(sfr_system *s, const DevSell &d, cudaStream_t st);

// kernels / solvers (krylov.cu)
int solve_device(sfr_system *s, int32_t solver, int32_t k, const double *d_diag_k,
                 const double *d_b, double *d_x, double tol, uint32_t maxit,
                 int32_t newx, int32_t precision, cudaStream_t st,
                 sfr_solve_info *info);
// FP32 inner Krylov with FP64 reliable updates (mixed.cu)
int solve_mixed(sfr_system *s, int32_t solver, int32_t k, const double *d_diag_k,
                const double *d_b, double *d_x, double tol, uint32_t maxit, int32_t newx,
                cudaStream_t st, sfr_solve_info *info);
// Batched (team) persistent launches, K = 1 (krylov.cu, mixed.cu)
struct TeamTable;
struct SolveOut;
size_t team_ws_bytes_fp64(int n, int grid);
size_t team_ws_bytes_mixed(int n, int grid);
int team_max_grid_fp64(int32_t solver, int device);
int team_max_grid_mixed(int32_t solver, int device);
int enqueue_team_fp64(sfr_system *s, int32_t solver, const double *d_b, double *d_x, double tol,
                      uint32_t maxit, int32_t newx, const TeamTable &team, int grid, void *ws,
                      SolveOut *d_out, unsigned *ctl, cudaStream_t st);
int enqueue_team_mixed(sfr_system *s, int32_t solver, const double *d_b, double *d_x, double tol,
                       uint32_t maxit, int32_t newx, const TeamTable &team, int grid, void *ws,
                       SolveOut *d_out, unsigned *ctl, cudaStream_t st);

// Resident engine (resident.cu): mixed PCG, one right-hand side, the
// system's own diagonal.  resident_fits: the pattern and size allow it;
// solve_resident returns SFR_UNSUPPORTED when the diagonal is not positive.
// Self-tests of the bounded device-side waits (sfr_gpu_wait_selftest):
// kind 0 grid_sync, 1 the fused iteration's tagged exchange; the resident
// engine's exchange.
int wait_selftest_fused(int32_t kind, int32_t absent, uint32_t spin_limit, cudaStream_t st);
int wait_selftest_resident(int32_t absent, uint32_t spin_limit, cudaStream_t st);
bool resident_fits(sfr_system *s);
int solve_resident(sfr_system *s, const double *d_b, double *d_x, double tol, uint32_t maxit,
                   int32_t newx, cudaStream_t st, sfr_solve_info *info);

// BiCGSTAB(2), GMRES(15), MINRES (krylov_ext.cu): one right-hand side, FP64;
// d_diag null means the system's own diagonal
int solve_ext(sfr_system *s, int32_t solver, const double *d_diag, const double *d_b, double *d_x,
              double tol, uint32_t maxit, int32_t newx, cudaStream_t st, sfr_solve_info *info);

// MINRES with its scalar recurrence on the device, one CUDA graph a solve
// (minres_graph.cu); d_diag null means the system's own diagonal
int solve_minres_graph(sfr_system *s, const double *d_diag, const double *d_b, double *d_x,
                       double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                       sfr_solve_info *info);
void release_minres_graph(const sfr_system *s);
// BiCGSTAB(2) the same way (bicgl2_graph.cu)
int solve_bicgstabl2_graph(sfr_system *s, const double *d_diag, const double *d_b, double *d_x,
                           double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                           sfr_solve_info *info);
void release_bicgstabl2_graph(const sfr_system *s);
int solve_gmres_graph(sfr_system *s, const double *d_diag, const double *d_b, double *d_x,
                      double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                      sfr_solve_info *info);
void release_gmres_graph(const sfr_system *s);

// Graph engine (stream_solve.cu)
int solve_stream(sfr_system *s, int32_t solver, int32_t k, const double *d_diag_k,
                 const double *d_b, double *d_x, double tol, uint32_t maxit, int32_t newx,
                 int32_t precision, double delta, int threads, int spw, int pf, int fused,
                 bool loop, cudaStream_t st, sfr_solve_info *info);
void release_stream_engine(const sfr_system *s);
double reliable_delta(int32_t solver);
double reliable_delta_resident();  // the resident engine's PCG factor
int spmv_device(sfr_system *s, const DevSell &A, const double *d_diag,
                const double *d_x, double *d_y, double *d_dot, cudaStream_t st);
int dot_device(const double *d_a, const double *d_b, int32_t n, double *d_dot,
               cudaStream_t st);
// (a, b) into host memory through the device's per-device scratch
int dot_host(const double *d_a, const double *d_b, int32_t n, double *h_out,
             cudaStream_t st);
int num_sms(int device);
// The autotuned choice for this kind of solve, or null (autotune.cpp).
const Tuned *find_tuned(const sfr_system *s, int32_t solver, int32_t k, int32_t precision,
                        bool own_diag);
// The automatic engine choice without a tuned entry: 1 persistent, 2 graph,
// 4 resident (krylov.cu).
int auto_engine(sfr_system *s, int32_t solver, int32_t k, int32_t precision, bool own_diag);
// Blocks of the standalone dot / SpMV+dot kernels (256 threads each) for n
// elements on `device`: 4 per SM of the device, at most one per 256 elements.
int stat_grid(int device, int64_t n);
// adjoint.cu: dJ/d(value source) and dJ/d(ad) from lam and x (device arrays)
int adjoint_gradients(sfr_system *s, const double *d_lam, const double *d_x, double *d_gsrc,
                      double *d_gad, cudaStream_t st);
// Text for sfr_last_error() (capi.cpp)
void set_last_error(const char *msg);
}  // namespace sfr
