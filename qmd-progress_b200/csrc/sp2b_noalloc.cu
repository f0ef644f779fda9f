// SP2 on one core+halo block without any memory allocation.
//
// Who needs this: code that must not call cudaMalloc (or any allocator) at the moment
// it wants a density block.  The usual case is a simulation code that claims its GPU
// memory up front through its own pool allocator and hands slices of it to the
// libraries it calls: a library allocation there either fails because the pool holds
// the memory, or breaks the pool's accounting.  Another is a time-step loop that may
// not stall on cudaMalloc / cudaFree, which synchronise the device.  Such callers pass
// their own device block (in/out) and host pp/vv; every working buffer this entry needs
// lives in the fixed device array below.
//
// Limits and sharing:
//  * block size n <= kNoAllocMaxN (512) and icount <= kNoAllocMaxIter (100, the size of
//    the reference's gp%pp / gp%vv, src/prg_graph_mod.F90:117-135); larger requests are
//    rejected with SP2B_BAD_ARG;
//  * the array (about 4.2 MB) is held by every GPU that loads this library until the
//    process exits;
//  * every call on a device uses the same array and leaves its contents behind; the
//    call clears what must start at zero itself.  Two calls whose GPU work overlaps
//    (different host threads, or different streams without ordering) race on it;
//  * the first call on a device looks up the array's device address (see
//    noalloc_scratch below); make that first call before any stream capture begins.
#include <cstring>
#include <mutex>

#include "kernels.cuh"

namespace sp2b {

constexpr int kNoAllocMaxN = 512;
constexpr int kNoAllocMaxIter = 100;
constexpr size_t kNoAllocSq = (size_t)kNoAllocMaxN * kNoAllocMaxN;  // padded block
constexpr int kNoAllocPartials = 4 * 148 * 8;                       // >= 4 x normalize grid

// Byte layout of the scratch array.
constexpr size_t kOffX0 = 0;
constexpr size_t kOffX1 = kOffX0 + kNoAllocSq * sizeof(double);
constexpr size_t kOffPart = kOffX1 + kNoAllocSq * sizeof(double);
constexpr size_t kOffRec = kOffPart + kNoAllocPartials * sizeof(double);
constexpr size_t kOffPP = kOffRec + ((kNoAllocMaxIter + 2) * sizeof(SP2Rec) + 255) / 256 * 256;
constexpr size_t kOffVV = kOffPP + ((kNoAllocMaxIter + 2) * sizeof(int) + 255) / 256 * 256;
constexpr size_t kOffSmall = kOffVV + ((kNoAllocMaxIter + 2) * sizeof(double) + 255) / 256 * 256;
constexpr size_t kOffCounter = kOffSmall + 16 * sizeof(double);
constexpr size_t kOffSout = kOffCounter + 256;
constexpr size_t kOffErr = kOffSout + 256;
constexpr size_t kNoAllocBytes = kOffErr + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch on the current device.  In host code the name
// g_noalloc_scratch is only a host-side stand-in, never a device address, so it is
// looked up once per device with cudaGetSymbolAddress (with that device current).
static void* noalloc_scratch(int dev, cudaError_t* err) {
  static std::mutex mu;
  static void* addr[64] = {};
  static bool looked_up[64] = {};
  if (dev < 0 || dev >= 64) {
    *err = cudaErrorInvalidDevice;
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!looked_up[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      *err = e;
      return nullptr;
    }
    addr[dev] = p;
    looked_up[dev] = true;
  }
  *err = cudaSuccess;
  return addr[dev];
}

}  // namespace sp2b

using namespace sp2b;

extern "C" int sp2b_sp2_submatrix_inplace_noalloc(double* x_dev, int n, const int* pp,
                                                  int icount, double* vv, double mineval,
                                                  double maxeval, int core_size, void* stream) {
  if (!x_dev || n <= 0 || icount < 0 || (icount > 0 && (!pp || !vv)) || core_size < 0 ||
      core_size > n) {
    set_last_error("sp2b_sp2_submatrix_inplace_noalloc: bad argument (n=%d icount=%d core=%d)",
                   n, icount, core_size);
    return SP2B_BAD_ARG;
  }
  if (n > kNoAllocMaxN || icount > kNoAllocMaxIter) {
    set_last_error("sp2b_sp2_submatrix_inplace_noalloc: n=%d / icount=%d exceed the fixed "
                   "scratch limits n <= %d, icount <= %d",
                   n, icount, kNoAllocMaxN, kNoAllocMaxIter);
    return SP2B_BAD_ARG;
  }
  if (!(maxeval - mineval > 0.0)) {
    set_last_error("sp2b_sp2_submatrix_inplace_noalloc: maxeval must exceed mineval");
    return SP2B_BAD_ARG;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    set_last_error("no CUDA device available");
    return SP2B_NO_DEVICE;
  }
  cudaError_t se;
  unsigned char* base = static_cast<unsigned char*>(noalloc_scratch(dev, &se));
  if (!base) {
    set_last_error("cudaGetSymbolAddress failed: %s", cudaGetErrorString(se));
    return SP2B_CUDA_ERROR;
  }
  double* x[2] = {reinterpret_cast<double*>(base + kOffX0), reinterpret_cast<double*>(base + kOffX1)};
  double* partials = reinterpret_cast<double*>(base + kOffPart);
  SP2Rec* rec = reinterpret_cast<SP2Rec*>(base + kOffRec);
  int* pp_d = reinterpret_cast<int*>(base + kOffPP);
  double* vv_d = reinterpret_cast<double*>(base + kOffVV);
  double* small = reinterpret_cast<double*>(base + kOffSmall);
  unsigned* counter = reinterpret_cast<unsigned*>(base + kOffCounter);
  SolveOut* sout = reinterpret_cast<SolveOut*>(base + kOffSout);
  int* err = reinterpret_cast<int*>(base + kOffErr);
  cudaStream_t st = (cudaStream_t)stream;
  const int np = padded(n);

  // state that must start at zero (the array keeps the previous call's contents)
  SP2B_CUDA_TRY(cudaMemsetAsync(counter, 0, 4 * sizeof(unsigned), st));
  SP2B_CUDA_TRY(cudaMemsetAsync(sout, 0, sizeof(SolveOut), st));
  SP2B_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  const double bounds[2] = {mineval, maxeval};
  SP2B_CUDA_TRY(cudaMemcpyAsync(small, bounds, sizeof(bounds), cudaMemcpyHostToDevice, st));
  if (icount > 0) {
    SP2B_CUDA_TRY(cudaMemcpyAsync(pp_d, pp, icount * sizeof(int), cudaMemcpyHostToDevice, st));
    if (core_size > 0)
      SP2B_CUDA_TRY(cudaMemcpyAsync(vv_d, vv, icount * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  // X0 = (maxeval I - x)/(maxeval - mineval) into the padded scratch block
  SP2B_CUDA_TRY(launch_normalize_f64(x_dev, n, n, np, small, x[0], partials, counter, rec,
                                     small + 4, st));
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.np = np;
  a.ld = np;
  a.control = 1;
  a.ctl.algo = ALGO_SEQ;
  a.ctl.icount = icount;
  a.ctl.n = n;
  a.rec = rec;
  a.pp_in = pp_d;
  a.vv_out = core_size > 0 ? vv_d : nullptr;   // no core rows: vv gains nothing
  a.vv_accumulate = 1;
  a.core = core_size > 0 ? core_size : -1;
  a.sout = sout;
  a.partials = partials;
  a.counter = counter;
  a.err = err;
  for (int k = 0; k < icount; ++k) {
    a.k = k;
    a.A = a.B = a.E = x[k & 1];
    a.out = x[(k + 1) & 1];
    SP2B_CUDA_TRY(launch_sym_gemm_f64(a, st));
  }
  SP2B_CUDA_TRY(launch_finish_f64(x[icount & 1], np, n, 2.0, x_dev, n, st));
  SolveOut so;
  memset(&so, 0, sizeof(so));
  double norm[4] = {0.0, 0.0, 0.0, 0.0};
  if (icount > 0 && core_size > 0)
    SP2B_CUDA_TRY(cudaMemcpyAsync(vv, vv_d, icount * sizeof(double), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(&so, sout, sizeof(SolveOut), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(norm, small + 4, sizeof(norm), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  // the same checks as the regular entry: bounds as used, and ||X0||_F^2 of the
  // normalised block, which shows a NaN / Inf input even when no step runs
  if (!(norm[1] - norm[0] > 0.0) || !(norm[3] == norm[3]) || norm[3] > 1e300) {
    set_last_error("non-finite values in the input block or degenerate bounds (%g, %g)",
                   norm[0], norm[1]);
    return SP2B_BAD_INPUT;
  }
  if (so.status != SP2B_OK) {
    set_last_error("non-finite values during SP2");
    return so.status;
  }
  return SP2B_OK;
}
