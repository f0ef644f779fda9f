// Launch interfaces shared by the sp2b translation units.
#pragma once
#include <string>
#include <vector>

#include "sp2b_common.cuh"

namespace sp2b {

// Counts kernel launches issued by the library (diagnostics / bench).
void note_launch(int k = 1);
long long launch_count();
void set_launch_count(long long v);

// Outcome of a dense solve, written by the device.
struct SolveOut {
  int done;     // loop finished
  int nupd;     // number of X updates applied (final X lives in buffer nupd & 1)
  int status;   // SP2B_* code
  int iter;     // Fortran iteration count ("icount")
};

// Arguments of one symmetric-tile product launch (FP64 or split precision).
//   acc(m, n) = sum_k A[k][m] * B[k][n]   (A, B stored np x np, symmetric)
//   out       = alpha * acc + beta * E     (upper tiles computed, mirrored on store)
// In control mode (ctl/rec set) alpha/beta come from the SP2 branch rule.
struct StepArgs {
  const void* A;
  const void* B;
  const void* A_lo;     // split mode: lo halves of the operands
  const void* B_lo;
  const void* E;        // elementwise operand (FP64; or hi/lo pair in split mode)
  void* out;            // nullptr: sums only
  const void* E_lo;     // split mode: lo half of E
  void* out_lo;         // split mode: lo half of out
  int np;               // padded dimension of a dense solve
  int ld;               // row pitch of A/B/E/out (dense: np; batched parts: max padded size)
  int ntiles;
  // Batched parts (tiles != nullptr): CTA b works on tile tiles[b] =
  //   {x: first packed row of its part, y: (bi << 16) | bj, z: padded part size, w: core rows}
  const int4* tiles;
  double alpha, beta;
  int core;             // > 0: residual sums over the first `core` rows only
  // SP2 control (control = 1)
  int control;
  SP2Ctl ctl;
  SP2Rec* rec;
  int k;
  const int* pp_in;
  int* pp_out;
  double* vv_out;
  int vv_accumulate;    // 1: vv_out[k] += res (submatrix); 0: vv_out[k] = sqrt(res)
  SolveOut* sout;
  // reductions
  double* partials;     // [ntiles][4]
  unsigned* counter;
  double* sums_out;     // non-control: the 4 totals {||out||^2, Tr out, ||E-acc||^2, Tr acc}
  int* err;             // device error word (timeouts)
  int n_out, ld_out;    // McWeeny combine: the n_out x n_out density and its row pitch
};

// FP64 path ---------------------------------------------------------------------------
int f64_tile(int np);  // tile edge chosen for this size (64 or 128)
std::string f64_tune_key(int np);
int tune_f64_tile(int np, const double* x_in, double* x_out, double* partials, unsigned* counter,
                  double* sums_out, cudaStream_t st);
int device_sms();       // SM count of the current device
int f64_ntiles(int np);
cudaError_t launch_gersh(const double* h, int n, int ld, double* rowsum, int nsplit,
                         double* bounds, double* partials, unsigned* counter, cudaStream_t st);
int gersh_nsplit(int n);
cudaError_t launch_normalize_f64(const double* h, int n, int ld, int np, const double* bounds,
                                 double* x, double* partials, unsigned* counter, SP2Rec* rec0,
                                 double* norm_out, cudaStream_t st);
cudaError_t launch_sym_gemm_f64(const StepArgs& a, cudaStream_t st);
cudaError_t launch_sym_gemm_f64_batched(const StepArgs& a, int bt, cudaStream_t st);

// All maxiter SP2 steps of a small batch of parts (the FP64 re-solve of flagged parts)
// in one cooperative launch: one CTA per 32 x 32 upper tile; the tiles of a part meet
// at a per-part barrier (a counter in `bar`, bounded wait) between steps.
struct MultiStepArgs {
  double* x[2];          // ping-pong packed buffers; x[0] holds X_0
  const int4* tiles;     // (row0, bi << 16 | bj, k extent, part)
  int ntiles;
  const int* part_tiles; // tiles per part
  const int* pp;         // device, maxiter branches (0: 2X - X^2, 1: X^2)
  int maxiter;
  int ld;
  unsigned* bar;         // one zeroed counter per part
  int* err;              // set to 1 when a barrier wait runs out
};
// Returns cudaErrorCooperativeLaunchTooLarge when the tiles cannot all be resident.
cudaError_t launch_f64_multistep(const MultiStepArgs& a, cudaStream_t st);
cudaError_t launch_finish_f64(const double* x, int np, int n, double scale, double* rho,
                              int ld, cudaStream_t st);
cudaError_t launch_copy_in(const double* src, int n, int ld, int np, double* x,
                           cudaStream_t st);
cudaError_t launch_mirror_lower(double* a, int n, int ld, cudaStream_t st);
cudaError_t launch_resp_init(const double* h1, int n, int ld, int np, const double* bounds,
                             double* d, cudaStream_t st);

// Split-precision (tcgen05) path ------------------------------------------------------
int tc_ntiles(int np);
cudaError_t launch_normalize_split(const double* h, int n, int ld, int np,
                                   const double* bounds, __half* hi, __half* lo, int bf16,
                                   double* partials, unsigned* counter, SP2Rec* rec0,
                                   double* norm_out, cudaStream_t st);
cudaError_t launch_sym_gemm_tc(const StepArgs& a, int bf16, cudaStream_t st);
// {G, X} = G X + X G of symmetric split matrices (A = G, B = X) on the upper tiles in one
// pass over the concatenated K range; out = alpha {G, X} + beta E.  FP16 split only;
// cudaErrorNotSupported unless np is a multiple of 256.
cudaError_t launch_anti_tc(const StepArgs& a, cudaStream_t st);
// batched parts: A/B tensors are rows x ld packed buffers
cudaError_t launch_sym_gemm_tc_batched(const StepArgs& a, long long rows, int bf16,
                                       cudaStream_t st);
cudaError_t launch_split_to_f64(const __half* hi, const __half* lo, int np, int bf16,
                                double* x, cudaStream_t st);
cudaError_t launch_wait_selftest(uint32_t limit, int* err, cudaStream_t st);
cudaError_t launch_f32_rows_to_split(const float* a, int m, int n, int mp, int np, __half* hi,
                                     __half* lo, cudaStream_t st);
cudaError_t launch_tc_panel(const __half* ahi, const __half* alo, int mp, const __half* bhi,
                            const __half* blo, int np, float* c, int m, int n, cudaStream_t st,
                            int* err);
cudaError_t launch_f32_to_split(const float* a, int n, int np, __half* hi, __half* lo,
                                cudaStream_t st);
cudaError_t launch_mcweeny_tc(const __half* xhi, const __half* xlo, const __half* rhi,
                              const __half* rlo, const double* x2, int np, int bf16, double* d,
                              int n, int ldd, double* partials, unsigned* counter,
                              double* sums_out, int* err, cudaStream_t st);

// INT8 (Ozaki residue) refinement products -------------------------------------------
int oz_nmod();
size_t oz_scale_bytes();
void oz_tile_list(int np, std::vector<int2>& out);
cudaError_t launch_oz_planes(const __half* xhi, const __half* xlo, int np, int bf16,
                             void* scale, int8_t* res, cudaStream_t st);
// SP2-step context of the launches that compute one step's X^2 in the exact INT8 mode.
struct OzStepCtl {
  const SolveOut* sout;
  const SP2Rec* rec;
  const int* pp_in;
  SP2Ctl ctl;
  int k;
  int active;   // 0: not part of an SP2 step (the McWeeny refinement)
};
cudaError_t launch_oz_gemm(const int8_t* res, int np, uint8_t* qout, const int2* tiles,
                           int ntiles, int* err, cudaStream_t st, const OzStepCtl* ctl = nullptr);
cudaError_t launch_oz_planes_f64(const double* x, int np, void* scale, int8_t* res,
                                 const OzStepCtl* ctl, cudaStream_t st);
cudaError_t launch_oz_crt_step(const uint8_t* q, const void* scale, const StepArgs& a,
                               cudaStream_t st);
cudaError_t launch_oz_crt(const uint8_t* q, const __half* xhi, const __half* xlo, int np,
                          int bf16, const void* scale, double* x2, __half* rhi, __half* rlo,
                          cudaStream_t st);
cudaError_t oz_read_scale(const void* scale, int* S, double* r2max, cudaStream_t st);
cudaError_t launch_tc_plain(const __half* ahi, const __half* alo, const __half* bhi,
                            const __half* blo, int np, float* c, int n, cudaStream_t st,
                            int* err);

}  // namespace sp2b
