// Launch interfaces of the graph-partitioned SP2 path.
#pragma once
#include "kernels.cuh"

namespace sp2b {

// One core+halo part inside the packed buffers.
struct PartDesc {
  long long row0;   // first packed row
  long long hoff;   // offset of its node list in the halo / sorted arrays
  long long coff;   // offset of its ncore x n block in the packed core-row output
  int n;            // core+halo size (lsize)
  int np;           // n padded to 128
  int ncore;        // core size (llsize)
  int pad_;
};

cudaError_t launch_extract_csr(const long long* rp, const int* col, const double* val,
                               const PartDesc* parts, int nparts, const int* halo,
                               const int* skey, const int* sval, int ld, double* xs,
                               cudaStream_t st);
cudaError_t launch_norm_parts(double* xs, const int* row_part, const PartDesc* parts,
                              long long rows, int ld, double emin, double emax, int prec,
                              void* hi, void* lo, cudaStream_t st);
cudaError_t launch_scatter_parts(const double* x64, const void* hi, const void* lo, int prec,
                                 const PartDesc* parts, int nparts, const int* halo, int ld,
                                 double* core_out, double* dense, long long n, cudaStream_t st);

// CSR extraction and normalisation with the global bounds in one pass (np <= 512 per
// part): split precisions into the packed hi/lo buffers, FP64 into xs.
cudaError_t launch_extract_split(const long long* rp, const int* col, const double* val,
                                 const PartDesc* parts, int nparts, const int* halo,
                                 const int* skey, const int* sval, int ld, double emin,
                                 double emax, int prec, void* hi, void* lo, double* xs,
                                 cudaStream_t st);

// Sum over each part's core rows of (X - X^2)_ii from the split iterate (hi, lo), as
// kPartIdemGroups partial sums per part (out[part * kPartIdemGroups + g]).
constexpr int kPartIdemGroups = 16;
cudaError_t launch_part_idem(const void* hi, const void* lo, int prec, const PartDesc* parts,
                             int nparts, int ld, double* out, cudaStream_t st);

cudaError_t launch_place_core(const long long* hptr, const int* halo, const int* lls,
                              const long long* off, int nparts, const double* src, double* rho,
                              long long n, cudaStream_t st);

// Batched INT8 digit-split form (exact INT8 precision of the sub-graph loop): the
// iterate as four signed 8-bit planes of M = rint(2^31 (X - I/2)) in each packed buffer
// (plane s at base + s rows ld).  Tiles {row0, bi << 16 | bj64, K extent, core} of
// 128 x 64 over the upper band of each part's block.  All steps run in one persistent
// launch; vv[k] += the core-row ||X_k - X_k^2||_F^2 of step k.
struct I8StepsArgs {
  const int4* tiles;
  const int* tpart;     // part of each tile
  const int* pnt;       // tiles of each part
  const int* pp;        // branch of each step: 0 = 2X - X^2, else X^2
  unsigned* done;       // per part, finished tiles over all steps (zero at launch)
  double* partials;     // step sums per (step, CTA, epilogue warp): i8_steps_partials (zero)
  int* err;
  int ntiles, nsteps, rows;
};
size_t i8_steps_partials(int nsteps);   // doubles
cudaError_t launch_i8_steps(const I8StepsArgs& a, const void* buf0, const void* buf1, int ld,
                            double* vv, cudaStream_t st);
cudaError_t launch_extract_digits(const long long* rp, const int* col, const double* val,
                                  const PartDesc* parts, int nparts, const int* halo,
                                  const int* skey, const int* sval, int ld, long long rows,
                                  double emin, double emax, int8_t* dig, cudaStream_t st);
cudaError_t launch_norm_digits(const double* xs, const int* row_part, const PartDesc* parts,
                               long long rows, int ld, double emin, double emax, int8_t* dig,
                               cudaStream_t st);
cudaError_t launch_scatter_digits(const int8_t* dig, long long rows, const PartDesc* parts,
                                  int nparts, const int* halo, int ld, double* core_out,
                                  double* dense, long long n, cudaStream_t st);
cudaError_t launch_part_idem_digits(const int8_t* dig, long long rows, const PartDesc* parts,
                                    int nparts, int ld, double* out, cudaStream_t st);

}  // namespace sp2b
