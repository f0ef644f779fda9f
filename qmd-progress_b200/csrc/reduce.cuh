// Deterministic block / grid reductions and the last-CTA SP2 finalisation.
#pragma once
#include "kernels.cuh"

namespace sp2b {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum NS values per thread over the block; result valid in thread 0.  Fixed
// shuffle/warp order, so the result is bitwise reproducible.
template <int NS>
__device__ __forceinline__ void block_sum(double (&v)[NS], double* red /*[32][NS]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NS; ++q) v[q] = warp_sum(v[q]);
  if (lane == 0)
    for (int q = 0; q < NS; ++q) red[warp * NS + q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < NS; ++q) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += red[w * NS + q];
      v[q] = s;
    }
  }
  __syncthreads();
}

// Publishes this CTA's 4 partial sums and, in the last CTA to arrive, reduces all
// partials in tile order and applies the SP2 control update for the next launch.
// No CTA waits on another: the last arrival does the work ("threadfence reduction").
__device__ inline void publish_and_finalize(const StepArgs& p, double (&s)[4], double* red,
                                            int* s_flag) {
  if (!p.partials) return;   // a product whose sums nobody reads (uniform over the grid)
  block_sum<4>(s, red);
  if (threadIdx.x == 0) {
    double* part = p.partials + 4 * (size_t)blockIdx.x;
    for (int q = 0; q < 4; ++q) part[q] = s[q];
    __threadfence();
    const unsigned ticket = atomicAdd(p.counter, 1u);
    *s_flag = (ticket == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!*s_flag) return;
  __threadfence();
  double t[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x)
    for (int q = 0; q < 4; ++q) t[q] += __ldcg(p.partials + 4 * (size_t)j + q);
  block_sum<4>(t, red);
  if (threadIdx.x != 0) return;
  *p.counter = 0u;
  if (p.control != 1) {
    if (p.sums_out)
      for (int q = 0; q < 4; ++q) p.sums_out[q] = t[q];
    return;
  }
  const SP2Rec r = p.rec[p.k];
  SP2Decision d = sp2_decide(p.ctl, r, p.k, p.pp_in);
  SP2Rec nx = d.next;
  if (p.ctl.algo == ALGO_MIXED) sp2_mixed_stop(p.ctl, r, t[3], nx);
  nx.fro2 = t[0];
  nx.trx_data = t[1];
  nx.trp = t[3];
  nx.pbias = r.fro2 - t[3];
  nx.last_branch = d.branch;
  if (p.pp_out) p.pp_out[p.k] = d.branch;
  if (p.vv_out) {
    if (p.vv_accumulate) p.vv_out[p.k] += t[2];
    else p.vv_out[p.k] = sqrt(t[2]);
  }
  if (!(t[0] == t[0]) || !(t[1] == t[1]) || !(t[2] == t[2]) || t[0] > 1e300) {
    nx.status = SP2B_BAD_INPUT;
    nx.done = 1;
  }
  if (p.err && *(volatile int*)p.err != 0) {
    nx.status = SP2B_TIMEOUT;
    nx.done = 1;
  }
  p.rec[p.k + 1] = nx;
  p.sout->nupd = p.k + 1;
  p.sout->iter = nx.iter;
  p.sout->status = nx.status;
  if (nx.done) p.sout->done = 1;
}

// Handles the start of a control-mode launch.  Returns the branch to apply, or -1 if
// this launch has nothing to do (loop already finished or stopping before update).
// Follower launches (control 2, 3: the products of the forward-mode response that run
// after step k) apply the branch that step k applied, and nothing when step k applied
// none: step k's last CTA recorded the update count (k + 1) and the branch in rec[k+1].
// (Reading the done word instead would drop the last update, whose record also ends the
// loop.)  They write no record.
__device__ inline int follow_branch(const StepArgs& p) {
  if (*(volatile const int*)&p.sout->nupd != p.k + 1) return -1;
  const int b = p.rec[p.k + 1].last_branch;
  return (b == BR_X2 || b == BR_2X_MINUS_X2) ? b : -1;
}

__device__ inline int control_prologue(const StepArgs& p) {
  if (p.control >= 2) return follow_branch(p);
  // The solve-wide done word is set by the launch that finished the loop; every
  // later launch of the same solve (the host launches in chunks) returns at once.
  if (*(volatile const int*)&p.sout->done) return -1;
  const SP2Rec r = p.rec[p.k];
  if (r.done) {
    // Reached at k = 0 when normalisation flagged the input.
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      p.rec[p.k + 1] = r;
      p.sout->nupd = p.k;
      p.sout->iter = r.iter;
      p.sout->status = r.status;
      p.sout->done = 1;
    }
    return -1;
  }
  SP2Decision d = sp2_decide(p.ctl, r, p.k, p.pp_in);
  if (d.branch == BR_STOP) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      SP2Rec nx = d.next;
      nx.done = 1;
      nx.last_branch = BR_STOP;
      p.rec[p.k + 1] = nx;
      p.sout->nupd = p.k;
      p.sout->iter = nx.iter;
      p.sout->status = nx.status;
      p.sout->done = 1;
    }
    return -1;
  }
  return d.branch;
}

__device__ __forceinline__ void upper_tile(int id, int& bi, int& bj) {
  int j = (int)((sqrt(8.0 * id + 1.0) - 1.0) * 0.5);
  while ((j + 1) * (j + 2) / 2 <= id) ++j;
  while (j * (j + 1) / 2 > id) --j;
  bj = j;
  bi = id - j * (j + 1) / 2;
}

// Weight of element (r, c) of an upper tile in the full-matrix sums: off-diagonal
// tiles stand for themselves and their mirror; in diagonal tiles only r <= c counts.
__device__ __forceinline__ int sym_weight(bool diag, int r, int c) {
  return diag ? (r < c ? 2 : (r == c ? 1 : 0)) : 2;
}
__device__ __forceinline__ int core_weight(int w, int r, int c, int core) {
  if (core <= 0 || w == 0) return w;
  if (r == c) return r < core ? 1 : 0;
  return (r < core ? 1 : 0) + (c < core ? 1 : 0);
}

}  // namespace sp2b
