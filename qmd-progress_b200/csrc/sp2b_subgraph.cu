// Host side of the graph-partitioned SP2 path: prg_subgraphSP2Loop
// (src/prg_subgraphloop_mod.F90:36-126) as one batched GPU solve.
//
// All parts share the branch sequence pp(1:maxIter) and the global bounds
// (src/prg_subgraphloop_mod.F90:104-106), so every part advances in lock step: one
// launch per SP2 iteration covers the upper tiles of every part (a ragged batch,
// largest parts first), and the whole sequence normalise -> maxIter steps -> scatter
// is captured once into a CUDA graph and replayed as one graph launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "kernels_subgraph.cuh"
#include "sp2b_ctx.h"
#include "sp2b_tune.h"

namespace sp2b {

template <typename T>
static cudaError_t grow_buf(T*& p, size_t& cap, size_t need) {
  if (need <= cap && p) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(need, 1) * sizeof(T));
  if (e == cudaSuccess) cap = std::max<size_t>(need, 1);
  return e;
}

// Page-locked host staging (the per-call readbacks leave in one copy batch and one wait).
template <typename T>
static cudaError_t grow_pinned(T*& p, size_t& cap, size_t need) {
  if (need <= cap && p) return cudaSuccess;
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMallocHost((void**)&p, std::max<size_t>(need, 1) * sizeof(T));
  if (e == cudaSuccess) cap = std::max<size_t>(need, 1);
  return e;
}

// 1 in *flag when the caller's part lists (halo_ptr, llsize) differ from the cached
// layout's (node-list offsets and core sizes per part, the total node count).
__global__ void k_cmp_parts(const long long* __restrict__ hp, const int* __restrict__ lls,
                            const PartDesc* __restrict__ parts, int nparts, long long nhalo,
                            int* flag) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= nparts; p += gridDim.x * blockDim.x) {
    const bool diff = p == nparts ? hp[p] != nhalo
                                  : (hp[p] != parts[p].hoff || lls[p] != parts[p].ncore);
    if (diff) *flag = 1;
  }
}

// ... and when the node lists differ; runs after k_cmp_parts and reads nothing of the
// caller's node list unless the counts agreed (it then has nhalo entries).
__global__ void k_cmp_halo(const int* __restrict__ hidx, const int* __restrict__ cached,
                           long long nhalo, int* flag) {
  if (*(volatile int*)flag) return;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nhalo;
       q += (long long)gridDim.x * blockDim.x)
    if (hidx[q] != cached[q]) *flag = 1;
}

struct SubBufs {
  double* xs = nullptr;          size_t xs_cap = 0;     // FP64 packed (H_sub / FP64 iterate)
  double* x2 = nullptr;          size_t x2_cap = 0;     // FP64 ping-pong partner
  __half* hi[2] = {};            size_t hi_cap[2] = {};
  __half* lo[2] = {};            size_t lo_cap[2] = {};
  int8_t* dig[2] = {};           size_t dig_cap[2] = {};   // INT8 digit planes (4 per buffer)
  int* tpart = nullptr;          size_t tpart_cap = 0;     // INT8: part of each tile
  double* i8part = nullptr;      size_t i8part_cap = 0;    // INT8: per-step sums
  PartDesc* parts = nullptr;     size_t parts_cap = 0;
  int4* tiles = nullptr;         size_t tiles_cap = 0;
  int* row_part = nullptr;       size_t row_part_cap = 0;
  int* halo = nullptr;           size_t halo_cap = 0;
  int* skey = nullptr;           size_t skey_cap = 0;
  int* sval = nullptr;           size_t sval_cap = 0;
  long long* rp = nullptr;       size_t rp_cap = 0;
  int* col = nullptr;            size_t col_cap = 0;
  double* val = nullptr;         size_t val_cap = 0;
  double* core = nullptr;        size_t core_cap = 0;
  double* dense = nullptr;       size_t dense_cap = 0;
  double* partials = nullptr;    size_t partials_cap = 0;
  SP2Rec* rec = nullptr;         size_t rec_cap = 0;
  int* pp = nullptr;             size_t pp_cap = 0;
  double* vv = nullptr;          size_t vv_cap = 0;
  double* idem = nullptr;        size_t idem_cap = 0;   // per-part core idempotency sums
  // 32-edge FP64 layouts: the tile list of the one-launch multi-step solve (the INT8
  // solve uses ms_part_tiles and ms_bar too: tiles per part, finished-tile counters)
  int4* ms_tiles = nullptr;      size_t ms_tiles_cap = 0;
  int* ms_part_tiles = nullptr;  size_t ms_part_tiles_cap = 0;
  unsigned* ms_bar = nullptr;    size_t ms_bar_cap = 0;
  int ms_ntiles = 0;
  double* hback = nullptr;       size_t hback_cap = 0;  // pinned: vv, part sums, status
  int* dflag = nullptr;          size_t dflag_cap = 0;  // device: part-list comparison
  // layout of the last call (reused when the part lists are unchanged)
  std::vector<long long> last_hp, last_coff;
  std::vector<int> last_lls, last_hidx, last_pp;
  const int* last_pp_dev = nullptr;
  std::vector<PartDesc> P;
  int ld = 0, ntiles = 0, layout_bt = 0, layout_order = 0, layout_dig = 0;
  long long rows = 0, coff = 0;
  bool layout_valid = false;
  // instantiated graph of the last call and the inputs it was captured with
  cudaGraphExec_t exec = nullptr;
  std::vector<unsigned char> exec_key;
};
static SubBufs g_sub[64];
static SubBufs g_sub_ref[64];  // the FP64 re-solve of the parts a split call flags

// True for page-locked (pinned or registered) host memory, which a copy on another
// stream can fill while kernels run.
static bool host_locked(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// A second stream per device for output copies that overlap the FP64 re-solve.
static cudaError_t copy_stream(int dev, cudaStream_t* s) {
  static cudaStream_t streams[64] = {};
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!streams[dev]) {
    const cudaError_t e = cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
  }
  *s = streams[dev];
  return cudaSuccess;
}

// Parts of the last sub-graph call of this thread solved again in FP64, and every
// part's core-row idempotency sum.
static thread_local std::vector<int> t_refined;
static thread_local std::vector<double> t_idem;

// One batched solve: the part lists are host vectors, H (CSR) and the outputs device
// arrays.  Stream-ordered on `st`; returns after the solve is complete.
struct SubJob {
  int n;
  const long long* rp;
  const int* col;
  const double* val;
  const std::vector<long long>* hp;
  const std::vector<int>* lls;
  const std::vector<int>* hidx;
  const int* pp;         // host, maxiter entries
  int maxiter;
  double mineval, maxeval;
  int prec;              // SP2B_PREC_FP64 / _MIXED_FP16 / _MIXED_BF16 / _EXACT_INT8
  double* core;          // device, packed core rows, or null
  double* dense;         // device, n x n, or null
  bool clear_dense;      // zero `dense` before the scatter
  bool part_idem;        // split and INT8 only: per-part idempotency sums into b.idem
  bool multistep;        // FP64 only: all steps in one cooperative launch when it fits
  // measured launch configuration (-1: the built-in rule).  FP64: the tile edge (32 or 64);
  // split: the order of the tile list (0 largest parts first, 1 balanced over the CTAs)
  int variant = -1;
  // per part, the offset of its ncore x n block in `core` (null: packed in part order)
  const std::vector<long long>* coff_at = nullptr;
  // part_idem: receives the per-part sums (nparts x kPartIdemGroups) with the vv readback
  std::vector<double>* idem_out = nullptr;
};

// Builds (or reuses) the layout, buffers and CUDA graph of `j` in `b`, launches the
// graph on `st` and waits for it.  vvh receives the per-iteration sums of squares.
static int batched_solve(Ctx* c, SubBufs& b, const SubJob& j, cudaStream_t st,
                         std::vector<double>& vvh) {
  const std::vector<long long>& hp = *j.hp;
  const std::vector<int>& lls = *j.lls;
  const std::vector<int>& hidx = *j.hidx;
  const int nparts = (int)lls.size();
  const int maxiter = j.maxiter, n = j.n, prec = j.prec;
  // split: FP16 / BF16 hi + lo products; dig: INT8 digit-split products
  const bool dig = prec == SP2B_PREC_EXACT_INT8;
  const bool split = prec == SP2B_PREC_MIXED_FP16 || prec == SP2B_PREC_MIXED_BF16;
  const long long nhalo = hp[nparts];
  cudaStream_t cap = c->stream;

  // tile edge of the step kernel: 128 split; FP64 64, or 32 when the 64-tiles of all
  // parts would not fill the SMs once (a handful of parts, e.g. the re-solve of flagged
  // ones).  The FP64 sums run in the same k order for every edge, so the results agree
  // bit for bit.
  int bt = 128;
  if (!split && !dig) {
    long long t64 = 0;
    for (int p = 0; p < nparts; ++p) {
      const long long t = padded((int)(hp[p + 1] - hp[p])) / 64;
      t64 += t * (t + 1) / 2;
    }
    bt = (t64 < 148 || j.multistep) ? 32 : 64;
    if (!j.multistep && (j.variant == 32 || j.variant == 64)) bt = j.variant;
  }
  const int tile_order = (split && j.variant == 1) ? 1 : 0;
  // (the caller may pass the cached lists themselves, which then need no comparison)
  static const std::vector<long long> no_coff;
  const std::vector<long long>& coff_at = j.coff_at ? *j.coff_at : no_coff;
  const bool same_layout = b.layout_valid && b.layout_bt == bt && b.layout_order == tile_order &&
                           b.layout_dig == (dig ? 1 : 0) && (&b.last_hp == &hp || b.last_hp == hp) &&
                           (&b.last_lls == &lls || b.last_lls == lls) &&
                           (&b.last_hidx == &hidx || b.last_hidx == hidx) && b.last_coff == coff_at;
  if (!same_layout) {
    b.layout_valid = false;
    std::vector<PartDesc>& P = b.P;
    P.assign(nparts, PartDesc());
    int ld = 0;
    long long rows = 0, coff = 0;
    for (int p = 0; p < nparts; ++p) {
      const long long sz = hp[p + 1] - hp[p];
      if (sz <= 0 || sz > 32768 || lls[p] < 0 || lls[p] > sz) {
        set_last_error("part %d: bad sizes (lsize=%lld llsize=%d)", p, sz, lls[p]);
        return SP2B_BAD_ARG;
      }
      PartDesc& d = P[p];
      d.n = (int)sz;
      d.np = padded(d.n);
      d.ncore = lls[p];
      d.hoff = hp[p];
      d.row0 = rows;
      d.coff = j.coff_at ? coff_at[p] : coff;
      d.pad_ = 0;
      rows += d.np;
      coff += (long long)d.ncore * d.n;
      ld = std::max(ld, d.np);
    }
    for (long long q = 0; q < nhalo; ++q)
      if (hidx[q] < 0 || hidx[q] >= n) {
        set_last_error("halo index out of range at %lld", q);
        return SP2B_BAD_ARG;
      }
    if (rows > 0x7fffffffLL) {
      set_last_error("packed parts exceed 2^31 rows");
      return SP2B_BAD_ARG;
    }
    // sorted node lists per part for the CSR column lookup
    std::vector<int> skey(nhalo), sval(nhalo), ord;
    for (int p = 0; p < nparts; ++p) {
      const int m = P[p].n;
      ord.resize(m);
      std::iota(ord.begin(), ord.end(), 0);
      const int* h = hidx.data() + P[p].hoff;
      std::sort(ord.begin(), ord.end(), [h](int a, int b2) { return h[a] < h[b2]; });
      for (int i = 0; i < m; ++i) {
        skey[P[p].hoff + i] = h[ord[i]];
        sval[P[p].hoff + i] = ord[i];
      }
    }
    std::vector<int> row_part(rows);
    for (int p = 0; p < nparts; ++p)
      std::fill(row_part.begin() + P[p].row0, row_part.begin() + P[p].row0 + P[p].np, p);
    // tile list, most expensive parts first (cost of a tile ~ np)
    std::vector<int> order(nparts);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b2) { return P[a].np > P[b2].np; });
    std::vector<int4> tiles;
    for (int p : order) {
      // a part without core rows contributes to neither rho nor vv: no tiles
      if (P[p].ncore <= 0) continue;
      if (dig) {
        // 128 x 64 tiles that reach the diagonal or lie above it, inside the part size
        // rounded up to 64 (also the K extent)
        const int n64 = (P[p].n + 63) / 64 * 64;
        for (int bi = 0; bi * 128 < n64; ++bi)
          for (int bj = 2 * bi; bj * 64 < n64; ++bj)
            tiles.push_back(make_int4((int)P[p].row0, (bi << 16) | bj, n64, P[p].ncore));
        continue;
      }
      const int T = P[p].np / bt;
      for (int bj = 0; bj < T; ++bj)
        for (int bi = 0; bi <= bj; ++bi)
          // K runs only to the part size rounded up to 64: the rest of the padded
          // block is zero, so those k-blocks contribute nothing
          tiles.push_back(make_int4((int)P[p].row0, (bi << 16) | bj,
                                    std::min(P[p].np, (P[p].n + 63) / 64 * 64), P[p].ncore));
    }
    if (tiles.empty()) {
      set_last_error("no part has core rows");
      return SP2B_BAD_ARG;
    }
    const int ntiles = (int)tiles.size();
    if (tile_order == 1) {
      // balanced: CTA c of the persistent grid (G CTAs) takes tiles c, c + G, ...; reversing
      // every other wave of the cost-sorted list pairs each CTA's expensive tiles with cheap
      // ones (the tiles' costs fall along the list: parts largest first)
      const int G = std::min(ntiles, device_sms());
      for (int w0 = G; w0 < ntiles; w0 += 2 * G)
        std::reverse(tiles.begin() + w0, tiles.begin() + std::min(ntiles, w0 + G));
    }
    if (bt == 32) {
      // the multi-step launch: one CTA per tile, the part index in place of the core count
      std::vector<int4> ms;
      std::vector<int> per(nparts, 0);
      for (const int4& t : tiles) {
        const int p = row_part[t.x];
        ms.push_back(make_int4(t.x, t.y, t.z, p));
        ++per[p];
      }
      SP2B_CUDA_TRY(grow_buf(b.ms_tiles, b.ms_tiles_cap, ms.size()));
      SP2B_CUDA_TRY(grow_buf(b.ms_part_tiles, b.ms_part_tiles_cap, (size_t)nparts));
      SP2B_CUDA_TRY(grow_buf(b.ms_bar, b.ms_bar_cap, (size_t)nparts));
      SP2B_CUDA_TRY(cudaMemcpyAsync(b.ms_tiles, ms.data(), ms.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
      SP2B_CUDA_TRY(cudaMemcpyAsync(b.ms_part_tiles, per.data(), nparts * sizeof(int), cudaMemcpyHostToDevice, st));
      b.ms_ntiles = (int)ms.size();
    }
    if (dig) {
      // the persistent INT8 solve orders a part's steps by counting its finished tiles
      std::vector<int> tp(ntiles), per(nparts, 0);
      for (int t = 0; t < ntiles; ++t) {
        tp[t] = row_part[tiles[t].x];
        ++per[tp[t]];
      }
      SP2B_CUDA_TRY(grow_buf(b.tpart, b.tpart_cap, (size_t)ntiles));
      SP2B_CUDA_TRY(grow_buf(b.ms_part_tiles, b.ms_part_tiles_cap, (size_t)nparts));
      SP2B_CUDA_TRY(grow_buf(b.ms_bar, b.ms_bar_cap, (size_t)nparts));
      SP2B_CUDA_TRY(cudaMemcpyAsync(b.tpart, tp.data(), ntiles * sizeof(int), cudaMemcpyHostToDevice, st));
      SP2B_CUDA_TRY(cudaMemcpyAsync(b.ms_part_tiles, per.data(), nparts * sizeof(int), cudaMemcpyHostToDevice, st));
      SP2B_CUDA_TRY(cudaStreamSynchronize(st));
    }
    SP2B_CUDA_TRY(grow_buf(b.parts, b.parts_cap, nparts));
    SP2B_CUDA_TRY(grow_buf(b.tiles, b.tiles_cap, ntiles));
    SP2B_CUDA_TRY(grow_buf(b.row_part, b.row_part_cap, rows));
    SP2B_CUDA_TRY(grow_buf(b.halo, b.halo_cap, nhalo));
    SP2B_CUDA_TRY(grow_buf(b.skey, b.skey_cap, nhalo));
    SP2B_CUDA_TRY(grow_buf(b.sval, b.sval_cap, nhalo));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.parts, P.data(), nparts * sizeof(PartDesc), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.tiles, tiles.data(), ntiles * sizeof(int4), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.row_part, row_part.data(), rows * sizeof(int), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.halo, hidx.data(), nhalo * sizeof(int), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.skey, skey.data(), nhalo * sizeof(int), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.sval, sval.data(), nhalo * sizeof(int), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaStreamSynchronize(st));  // host staging vectors go out of scope
    b.ld = ld;
    b.rows = rows;
    b.coff = coff;
    b.ntiles = ntiles;
    if (&b.last_hp != &hp) b.last_hp = hp;
    if (&b.last_lls != &lls) b.last_lls = lls;
    if (&b.last_hidx != &hidx) b.last_hidx = hidx;
    b.last_coff = coff_at;
    b.layout_bt = bt;
    b.layout_order = tile_order;
    b.layout_dig = dig ? 1 : 0;
    b.layout_valid = true;
  }
  const int ld = b.ld;
  const long long rows = b.rows;
  const int ntiles = b.ntiles;

  // ---- device buffers ----
  const size_t packed = (size_t)rows * ld;
  // parts up to 512: CSR straight to X0 (split: hi/lo, no FP64 block; FP64: no clearing)
  const bool fused = ld <= 512;
  if ((!split && !dig) || !fused) SP2B_CUDA_TRY(grow_buf(b.xs, b.xs_cap, packed));
  if (split) {
    for (int i = 0; i < 2; ++i) {
      SP2B_CUDA_TRY(grow_buf(b.hi[i], b.hi_cap[i], packed));
      SP2B_CUDA_TRY(grow_buf(b.lo[i], b.lo_cap[i], packed));
    }
  } else if (dig) {
    for (int i = 0; i < 2; ++i) SP2B_CUDA_TRY(grow_buf(b.dig[i], b.dig_cap[i], 4 * packed));
    SP2B_CUDA_TRY(grow_buf(b.i8part, b.i8part_cap, i8_steps_partials(maxiter)));
  } else {
    SP2B_CUDA_TRY(grow_buf(b.x2, b.x2_cap, packed));
  }
  const bool idem = (split || dig) && j.part_idem;
  if (idem) SP2B_CUDA_TRY(grow_buf(b.idem, b.idem_cap, (size_t)nparts * kPartIdemGroups));
  SP2B_CUDA_TRY(grow_buf(b.partials, b.partials_cap, 4 * (size_t)ntiles));
  SP2B_CUDA_TRY(grow_buf(b.rec, b.rec_cap, (size_t)maxiter + 2));
  SP2B_CUDA_TRY(grow_buf(b.pp, b.pp_cap, (size_t)maxiter + 1));
  SP2B_CUDA_TRY(grow_buf(b.vv, b.vv_cap, (size_t)maxiter + 1));
  // pp is a host array in every mode; uploaded when it changed (or its buffer did)
  if (maxiter > 0 && (b.pp != b.last_pp_dev || (int)b.last_pp.size() != maxiter ||
                      !std::equal(b.last_pp.begin(), b.last_pp.end(), j.pp))) {
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.pp, j.pp, maxiter * sizeof(int), cudaMemcpyHostToDevice, st));
    b.last_pp.assign(j.pp, j.pp + maxiter);
    b.last_pp_dev = b.pp;
  }
  double* core_d = j.core;
  double* dense_d = j.dense;

  // ---- a few FP64 parts: every step in one cooperative launch ----
  if (j.multistep && !split && !dig && bt == 32 && maxiter > 0) {
    SP2B_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(int), st));
    SP2B_CUDA_TRY(cudaMemsetAsync(b.ms_bar, 0, nparts * sizeof(unsigned), st));
    if (dense_d && j.clear_dense)
      SP2B_CUDA_TRY(cudaMemsetAsync(dense_d, 0, (size_t)n * n * sizeof(double), st));
    if (fused) {
      SP2B_CUDA_TRY(launch_extract_split(j.rp, j.col, j.val, b.parts, nparts, b.halo, b.skey,
                                         b.sval, ld, j.mineval, j.maxeval, prec, nullptr, nullptr,
                                         b.xs, st));
    } else {
      SP2B_CUDA_TRY(cudaMemsetAsync(b.xs, 0, packed * sizeof(double), st));
      SP2B_CUDA_TRY(launch_extract_csr(j.rp, j.col, j.val, b.parts, nparts, b.halo, b.skey,
                                       b.sval, ld, b.xs, st));
      SP2B_CUDA_TRY(launch_norm_parts(b.xs, b.row_part, b.parts, rows, ld, j.mineval, j.maxeval,
                                      prec, nullptr, nullptr, st));
    }
    MultiStepArgs ma;
    ma.x[0] = b.xs;
    ma.x[1] = b.x2;
    ma.tiles = b.ms_tiles;
    ma.ntiles = b.ms_ntiles;
    ma.part_tiles = b.ms_part_tiles;
    ma.pp = b.pp;
    ma.maxiter = maxiter;
    ma.ld = ld;
    ma.bar = b.ms_bar;
    ma.err = c->err;
    const cudaError_t me = launch_f64_multistep(ma, st);
    if (me == cudaSuccess) {
      SP2B_CUDA_TRY(launch_scatter_parts((maxiter & 1) ? b.x2 : b.xs, nullptr, nullptr, prec,
                                         b.parts, nparts, b.halo, ld, core_d, dense_d, n, st));
      SP2B_CUDA_TRY(grow_pinned(b.hback, b.hback_cap, 1));
      SP2B_CUDA_TRY(cudaMemcpyAsync(b.hback, c->err, sizeof(int), cudaMemcpyDeviceToHost, st));
      SP2B_CUDA_TRY(cudaStreamSynchronize(st));
      int herr = 0;
      memcpy(&herr, b.hback, sizeof(int));
      if (herr) {
        set_last_error("a device-side wait timed out");
        return SP2B_TIMEOUT;
      }
      vvh.assign(maxiter + 1, 0.0);   // the one-launch form forms no per-step sums
      return SP2B_OK;
    }
    if (me != cudaErrorCooperativeLaunchTooLarge) {
      set_last_error("multi-step launch failed: %s", cudaGetErrorString(me));
      return SP2B_CUDA_ERROR;
    }
    (void)cudaGetLastError();   // too many tiles to be resident at once: per-step launches
  }

  // ---- the batched solve, captured once into a graph ----
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.ld = ld;
  a.np = ld;
  a.ntiles = ntiles;
  a.tiles = b.tiles;
  a.control = 1;
  a.ctl.algo = ALGO_SEQ;
  a.ctl.icount = maxiter;
  a.ctl.n = n;
  a.rec = b.rec;
  a.pp_in = b.pp;
  a.pp_out = nullptr;
  a.vv_out = b.vv;
  a.vv_accumulate = 1;
  a.sout = c->sout;
  a.partials = b.partials;
  a.counter = c->counter;
  a.err = c->err;

  // The captured graph bakes in every pointer, size and scalar it launches with;
  // reuse it when all of them are unchanged.
  struct Key {
    const void* p[25];
    long long q[10];
    double d[2];
  } key;
  memset(&key, 0, sizeof(key));
  const void* ptrs[25] = {j.rp, j.col, j.val, core_d, dense_d, b.xs, b.x2,
                          dig ? (const void*)b.dig[0] : b.hi[0], dig ? (const void*)b.dig[1] : b.hi[1],
                          b.lo[0], b.lo[1], b.parts, b.tiles, b.row_part, b.halo, b.skey,
                          b.sval, b.partials, b.rec, b.pp, (const void*)cap,
                          idem ? b.idem : nullptr, dig ? b.tpart : nullptr,
                          dig ? b.ms_bar : nullptr, dig ? b.i8part : nullptr};
  memcpy(key.p, ptrs, sizeof(ptrs));
  const long long qs[10] = {n, nparts, rows, ld, maxiter, prec, ntiles, (long long)(size_t)b.vv,
                            j.clear_dense ? 1 : 0, bt};
  memcpy(key.q, qs, sizeof(qs));
  key.d[0] = j.mineval;
  key.d[1] = j.maxeval;
  std::vector<unsigned char> kbytes((unsigned char*)&key, (unsigned char*)&key + sizeof(key));
  const bool reuse = b.exec && b.exec_key == kbytes;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = reuse ? b.exec : nullptr;
  if (!reuse) {
    if (b.exec) {
      cudaGraphExecDestroy(b.exec);
      b.exec = nullptr;
    }
    const long long launches_before = launch_count();  // captured launches do not run yet
    SP2B_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    auto body = [&]() -> cudaError_t {
      cudaError_t e;
      if (!fused && (e = cudaMemsetAsync(b.xs, 0, packed * sizeof(double), cap)) != cudaSuccess)
        return e;
      if ((e = cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), cap)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(c->err, 0, sizeof(int), cap)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(c->sout, 0, sizeof(SolveOut), cap)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(b.rec, 0, sizeof(SP2Rec), cap)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(b.vv, 0, ((size_t)maxiter + 1) * sizeof(double), cap)) != cudaSuccess)
        return e;
      if (dense_d && j.clear_dense &&
          (e = cudaMemsetAsync(dense_d, 0, (size_t)n * n * sizeof(double), cap)) != cudaSuccess)
        return e;
      if (dig) {
        // The steps write each part's tiles (rows to the 128-row block, columns to the part
        // size rounded up to 64).  The second buffer's other entries are not cleared: the
        // mirrored operand loads reach columns past the tiles only for rows past them, so
        // stale values there feed padding rows alone, which no core row, sum or scatter
        // reads.
        if (fused) {
          if ((e = launch_extract_digits(j.rp, j.col, j.val, b.parts, nparts, b.halo, b.skey,
                                         b.sval, ld, rows, j.mineval, j.maxeval, b.dig[0], cap)) !=
              cudaSuccess)
            return e;
        } else {
          if ((e = launch_extract_csr(j.rp, j.col, j.val, b.parts, nparts, b.halo, b.skey, b.sval,
                                      ld, b.xs, cap)) != cudaSuccess)
            return e;
          if ((e = launch_norm_digits(b.xs, b.row_part, b.parts, rows, ld, j.mineval, j.maxeval,
                                      b.dig[0], cap)) != cudaSuccess)
            return e;
        }
      } else if (fused) {
        if ((e = launch_extract_split(j.rp, j.col, j.val, b.parts, nparts, b.halo, b.skey, b.sval,
                                      ld, j.mineval, j.maxeval, prec, split ? b.hi[0] : nullptr,
                                      split ? b.lo[0] : nullptr, split ? nullptr : b.xs, cap)) !=
            cudaSuccess)
          return e;
      } else {
        if ((e = launch_extract_csr(j.rp, j.col, j.val, b.parts, nparts, b.halo, b.skey, b.sval,
                                    ld, b.xs, cap)) != cudaSuccess)
          return e;
        if ((e = launch_norm_parts(b.xs, b.row_part, b.parts, rows, ld, j.mineval, j.maxeval, prec,
                                   split ? (void*)b.hi[0] : nullptr,
                                   split ? (void*)b.lo[0] : nullptr, cap)) != cudaSuccess)
          return e;
      }
      if (dig && maxiter > 0) {
        // every step in one persistent launch
        if ((e = cudaMemsetAsync(b.ms_bar, 0, nparts * sizeof(unsigned), cap)) != cudaSuccess)
          return e;
        if ((e = cudaMemsetAsync(b.i8part, 0, i8_steps_partials(maxiter) * sizeof(double), cap)) !=
            cudaSuccess)
          return e;
        I8StepsArgs ia;
        ia.tiles = b.tiles;
        ia.tpart = b.tpart;
        ia.pnt = b.ms_part_tiles;
        ia.pp = b.pp;
        ia.done = b.ms_bar;
        ia.partials = b.i8part;
        ia.err = c->err;
        ia.ntiles = ntiles;
        ia.nsteps = maxiter;
        ia.rows = (int)rows;
        if ((e = launch_i8_steps(ia, b.dig[0], b.dig[1], ld, b.vv, cap)) != cudaSuccess) return e;
      }
      for (int k = 0; k < maxiter && !dig; ++k) {
        a.k = k;
        const int bin = k & 1, bout = (k + 1) & 1;
        if (split) {
          a.A = a.B = a.E = b.hi[bin];
          a.A_lo = a.B_lo = a.E_lo = b.lo[bin];
          a.out = b.hi[bout];
          a.out_lo = b.lo[bout];
          e = launch_sym_gemm_tc_batched(a, rows, prec == SP2B_PREC_MIXED_BF16, cap);
        } else {
          double* xin = bin ? b.x2 : b.xs;
          double* xout = bout ? b.x2 : b.xs;
          a.A = a.B = a.E = xin;
          a.out = xout;
          e = launch_sym_gemm_f64_batched(a, bt, cap);
        }
        if (e != cudaSuccess) return e;
      }
      const int fb = maxiter & 1;
      if (dig) {
        if ((e = launch_scatter_digits(b.dig[fb], rows, b.parts, nparts, b.halo, ld, core_d,
                                       dense_d, n, cap)) != cudaSuccess)
          return e;
        if (idem)
          return launch_part_idem_digits(b.dig[fb], rows, b.parts, nparts, ld, b.idem, cap);
        return cudaSuccess;
      }
      if ((e = launch_scatter_parts(fb ? b.x2 : b.xs, split ? (void*)b.hi[fb] : nullptr,
                                    split ? (void*)b.lo[fb] : nullptr, prec, b.parts, nparts,
                                    b.halo, ld, core_d, dense_d, n, cap)) != cudaSuccess)
        return e;
      if (idem)
        return launch_part_idem(b.hi[fb], b.lo[fb], prec, b.parts, nparts, ld, b.idem, cap);
      return cudaSuccess;
    };
    const cudaError_t be = body();
    const cudaError_t ce = cudaStreamEndCapture(cap, &graph);
    set_launch_count(launches_before);
    if (be != cudaSuccess || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      set_last_error("graph capture failed: %s / %s", cudaGetErrorString(be), cudaGetErrorString(ce));
      return SP2B_CUDA_ERROR;
    }
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      set_last_error("graph instantiate failed: %s", cudaGetErrorString(ie));
      return SP2B_CUDA_ERROR;
    }
    b.exec = exec;
    b.exec_key = kbytes;
  }
  cudaError_t le = cudaGraphLaunch(exec, st);
  // extract, normalise, the steps (INT8: one persistent launch and its sums), scatter
  note_launch((dig ? (fused ? 1 : 2) + (maxiter > 0 ? 2 : 0) + 1 : maxiter + 3) + (idem ? 1 : 0));
  if (le != cudaSuccess) {
    set_last_error("graph launch failed: %s", cudaGetErrorString(le));
    return SP2B_CUDA_ERROR;
  }
  // the sums, the part sums and the status leave together, then one wait
  const size_t nv = (size_t)maxiter;
  const size_t ni = (idem && j.idem_out) ? (size_t)nparts * kPartIdemGroups : 0;
  SP2B_CUDA_TRY(grow_pinned(b.hback, b.hback_cap, nv + ni + 1));
  if (nv) SP2B_CUDA_TRY(cudaMemcpyAsync(b.hback, b.vv, nv * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (ni)
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.hback + nv, b.idem, ni * sizeof(double), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(b.hback + nv + ni, c->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  vvh.assign(maxiter + 1, 0.0);
  std::copy(b.hback, b.hback + nv, vvh.begin());
  if (ni) j.idem_out->assign(b.hback + nv, b.hback + nv + ni);
  int herr = 0;
  memcpy(&herr, b.hback + nv + ni, sizeof(int));
  if (herr) {
    set_last_error("a device-side wait timed out");
    return SP2B_TIMEOUT;
  }
  for (int k = 0; k < maxiter; ++k)
    if (!(vvh[k] == vvh[k])) {
      set_last_error("non-finite values during sub-graph SP2");
      return SP2B_BAD_INPUT;
    }
  return SP2B_OK;
}

// The measured configuration of a batched solve (FP64: tile edge 64 or 32; split: tile
// order), chosen once per device, precision and multiset of padded part sizes by timing
// whole solves of this job; sets j.variant.
static int tune_subgraph(Ctx* c, SubBufs& b, SubJob& j, cudaStream_t st) {
  j.variant = -1;
  if (!tune_enabled() || j.multistep || j.prec == SP2B_PREC_EXACT_INT8) return SP2B_OK;
  const bool split = j.prec != SP2B_PREC_FP64;
  const std::vector<long long>& hp = *j.hp;
  std::map<int, int> hist;
  for (size_t p = 0; p + 1 < hp.size(); ++p) ++hist[padded((int)(hp[p + 1] - hp[p]))];
  std::string key = std::string("subgraph/") + (split ? "split" : "f64") + "/sm" +
                    std::to_string(device_sms()) + "/";
  for (const auto& kv : hist) key += std::to_string(kv.first) + "x" + std::to_string(kv.second) + ",";
  int choice = -1;
  if (tune_lookup(key, &choice)) {
    j.variant = choice;
    return SP2B_OK;
  }
  if (j.maxiter <= 0) return SP2B_OK;   // no steps to time
  const int cands[2] = {split ? 0 : 64, split ? 1 : 32};
  std::vector<double> vtmp;
  std::vector<float> ms;
  int best = 0;
  const int rc = tune_measure(2, 2, st, [&](int k) {
    SubJob jc = j;
    jc.variant = cands[k];
    return batched_solve(c, b, jc, st, vtmp);
  }, &ms, &best);
  if (rc != SP2B_OK) return rc;
  tune_store(key, cands[best], ms);
  j.variant = cands[best];
  return SP2B_OK;
}

}  // namespace sp2b

using namespace sp2b;

extern "C" int sp2b_subgraph_sp2_loop(int n, const long long* h_row_ptr, const int* h_col,
                                      const double* h_val, int nparts, const long long* halo_ptr,
                                      const int* halo_idx, const int* llsize, const int* pp,
                                      int maxiter, double mineval, double maxeval,
                                      double* rho_core, double* rho_dense, double* vv,
                                      const sp2b_opts* opts) {
  t_refined.clear();
  t_idem.clear();
  if (n <= 0 || nparts <= 0 || !h_row_ptr || !h_col || !h_val || !halo_ptr || !halo_idx ||
      !llsize || maxiter < 0 || (maxiter > 0 && !pp) || !(maxeval - mineval > 0.0)) {
    set_last_error("sp2b_subgraph_sp2_loop: bad argument");
    return SP2B_BAD_ARG;
  }
  sp2b_opts dflt;
  sp2b_opts_default(&dflt);
  dflt.precision = SP2B_PREC_MIXED_FP16;
  if (!opts) opts = &dflt;
  const int prec = opts->precision;
  if (prec != SP2B_PREC_FP64 && prec != SP2B_PREC_MIXED_FP16 && prec != SP2B_PREC_MIXED_BF16 &&
      prec != SP2B_PREC_EXACT_INT8) {
    set_last_error("sp2b_subgraph_sp2_loop: unknown precision %d", prec);
    return SP2B_BAD_ARG;
  }
  const bool dev = opts->device_ptrs != 0;
  const bool split = prec != SP2B_PREC_FP64;   // every non-FP64 form may re-solve parts
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  SubBufs& b = g_sub[c->dev];
  // work is ordered on the caller's stream (device pointers: NULL = the default
  // stream); the CUDA graph is captured on the library stream and launched on `st`
  cudaStream_t st = opts->stream ? (cudaStream_t)opts->stream : (dev ? (cudaStream_t)0 : c->stream);

  // ---- host-side layout (index lists are small) ----
  // Device inputs: when a layout is cached, the caller's lists are compared with it on the
  // device (two small kernels and one 4-byte readback, in stream order) and the cached host
  // copies are used when they agree; otherwise the lists are fetched.
  std::vector<long long> hp_own;
  std::vector<int> lls_own, hidx_own;
  const std::vector<long long>* php = &hp_own;
  const std::vector<int>* plls = &lls_own;
  const std::vector<int>* phidx = &hidx_own;
  bool cached = false;
  if (dev && b.layout_valid && (int)b.P.size() == nparts &&
      b.last_hp.size() == (size_t)nparts + 1) {
    SP2B_CUDA_TRY(grow_buf(b.dflag, b.dflag_cap, 1));
    SP2B_CUDA_TRY(grow_pinned(b.hback, b.hback_cap, 1));
    SP2B_CUDA_TRY(cudaMemsetAsync(b.dflag, 0, sizeof(int), st));
    const long long nh = b.last_hp[nparts];
    k_cmp_parts<<<nparts / 256 + 1, 256, 0, st>>>(halo_ptr, llsize, b.parts, nparts, nh, b.dflag);
    k_cmp_halo<<<(int)std::min<long long>(nh / 256 + 1, 4 * 148), 256, 0, st>>>(halo_idx, b.halo,
                                                                                nh, b.dflag);
    note_launch(2);
    SP2B_CUDA_TRY(cudaGetLastError());
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.hback, b.dflag, sizeof(int), cudaMemcpyDeviceToHost, st));
    SP2B_CUDA_TRY(cudaStreamSynchronize(st));
    int diff = 1;
    memcpy(&diff, b.hback, sizeof(int));
    cached = diff == 0;
  }
  if (cached) {
    php = &b.last_hp;
    plls = &b.last_lls;
    phidx = &b.last_hidx;
  } else {
    hp_own.resize(nparts + 1);
    lls_own.resize(nparts);
    if (dev) {
      SP2B_CUDA_TRY(cudaMemcpy(hp_own.data(), halo_ptr, (nparts + 1) * sizeof(long long),
                               cudaMemcpyDeviceToHost));
      SP2B_CUDA_TRY(cudaMemcpy(lls_own.data(), llsize, nparts * sizeof(int), cudaMemcpyDeviceToHost));
    } else {
      std::memcpy(hp_own.data(), halo_ptr, (nparts + 1) * sizeof(long long));
      std::memcpy(lls_own.data(), llsize, nparts * sizeof(int));
    }
    if (hp_own[nparts] < 0) {
      set_last_error("sp2b_subgraph_sp2_loop: bad halo_ptr");
      return SP2B_BAD_ARG;
    }
    hidx_own.resize(hp_own[nparts]);
    if (dev)
      SP2B_CUDA_TRY(cudaMemcpy(hidx_own.data(), halo_idx, hidx_own.size() * sizeof(int),
                               cudaMemcpyDeviceToHost));
    else
      std::memcpy(hidx_own.data(), halo_idx, hidx_own.size() * sizeof(int));
  }
  const std::vector<long long>& hp = *php;
  const std::vector<int>& lls = *plls;
  const std::vector<int>& hidx = *phidx;
  long long coff = 0;
  for (int p = 0; p < nparts; ++p) coff += (long long)lls[p] * (hp[p + 1] - hp[p]);

  // ---- H and the outputs on the device ----
  const long long* rp_d = h_row_ptr;
  const int* col_d = h_col;
  const double* val_d = h_val;
  if (!dev) {
    const long long nnz = h_row_ptr[n];
    SP2B_CUDA_TRY(grow_buf(b.rp, b.rp_cap, (size_t)n + 1));
    SP2B_CUDA_TRY(grow_buf(b.col, b.col_cap, (size_t)nnz));
    SP2B_CUDA_TRY(grow_buf(b.val, b.val_cap, (size_t)nnz));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.rp, h_row_ptr, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.col, h_col, nnz * sizeof(int), cudaMemcpyHostToDevice, st));
    SP2B_CUDA_TRY(cudaMemcpyAsync(b.val, h_val, nnz * sizeof(double), cudaMemcpyHostToDevice, st));
    rp_d = b.rp;
    col_d = b.col;
    val_d = b.val;
  }
  double* core_d = rho_core;
  double* dense_d = rho_dense;
  if (!dev) {
    if (rho_core) {
      SP2B_CUDA_TRY(grow_buf(b.core, b.core_cap, (size_t)coff));
      core_d = b.core;
    }
    if (rho_dense) {
      SP2B_CUDA_TRY(grow_buf(b.dense, b.dense_cap, (size_t)n * n));
      dense_d = b.dense;
    }
  }

  const bool refine = split && opts->refine_tol > 0.0 && maxiter > 0;
  bool core_out_done = false;   // the core rows already reached rho_core (host calls)
  SubJob j{n, rp_d, col_d, val_d, &hp, &lls, &hidx, pp, maxiter, mineval, maxeval, prec,
           core_d, dense_d, true, refine, false};
  std::vector<double> vvh, part;
  int rc = tune_subgraph(c, b, j, st);
  if (rc != SP2B_OK) return rc;
  j.idem_out = refine ? &part : nullptr;   // the part sums come back with vv
  rc = batched_solve(c, b, j, st, vvh);
  if (rc != SP2B_OK) return rc;

  // ---- FP64 re-solve of the parts left with a half-occupied state ----
  if (refine) {
    if (part.size() != (size_t)nparts * kPartIdemGroups) {
      set_last_error("sp2b_subgraph_sp2_loop: part sums missing");
      return SP2B_CUDA_ERROR;
    }
    t_idem.assign(nparts, 0.0);
    for (int p = 0; p < nparts; ++p)
      for (int g = 0; g < kPartIdemGroups; ++g) t_idem[p] += part[(size_t)p * kPartIdemGroups + g];
    std::vector<long long> rhp(1, 0);
    std::vector<int> rlls, ridx;
    for (int p = 0; p < nparts; ++p) {
      if (!(t_idem[p] > opts->refine_tol)) continue;
      t_refined.push_back(p);
      ridx.insert(ridx.end(), hidx.begin() + hp[p], hidx.begin() + hp[p + 1]);
      rhp.push_back((long long)ridx.size());
      rlls.push_back(lls[p]);
    }
    if (!t_refined.empty()) {
      SubBufs& rb = g_sub_ref[c->dev];
      // A host-pointer call whose core output is page-locked: the split solve's core rows
      // (final but for the re-solved parts' blocks) leave on a second stream while the
      // re-solve runs, and the re-solved blocks follow from its output once they are out.
      cudaStream_t cs = nullptr;
      if (!dev && rho_core && host_locked(rho_core)) {
        SP2B_CUDA_TRY(copy_stream(c->dev, &cs));
        SP2B_CUDA_TRY(cudaMemcpyAsync(rho_core, b.core, coff * sizeof(double),
                                      cudaMemcpyDeviceToHost, cs));
      }
      // Otherwise the re-solve writes each part's block in place in the core output (part
      // p's block sits at sum_{q<p} llsize[q] * lsize[q]); with the copy stream it writes
      // them packed into its own buffer, from which they follow the copy.
      std::vector<long long> rcoffs;
      double* rcore = nullptr;
      if (core_d && cs) {
        long long rcoff = 0;
        for (size_t q = 0; q < rlls.size(); ++q) rcoff += (long long)rlls[q] * (rhp[q + 1] - rhp[q]);
        SP2B_CUDA_TRY(grow_buf(rb.core, rb.core_cap, (size_t)std::max(rcoff, 1LL)));
        rcore = rb.core;
      } else if (core_d) {
        std::vector<long long> start(nparts + 1, 0);
        for (int p = 0; p < nparts; ++p) start[p + 1] = start[p] + (long long)lls[p] * (hp[p + 1] - hp[p]);
        for (const int p : t_refined) rcoffs.push_back(start[p]);
        rcore = core_d;
      }
      SubJob rj{n, rp_d, col_d, val_d, &rhp, &rlls, &ridx, pp, maxiter, mineval, maxeval,
                SP2B_PREC_FP64, rcore, dense_d, false, false, true};
      if (core_d && !cs) rj.coff_at = &rcoffs;
      std::vector<double> rvv;
      rc = batched_solve(c, rb, rj, st, rvv);
      if (cs) {
        const cudaError_t ce = cudaStreamSynchronize(cs);
        if (rc == SP2B_OK && ce != cudaSuccess) {
          set_last_error("core-row copy failed: %s", cudaGetErrorString(ce));
          return SP2B_CUDA_ERROR;
        }
      }
      if (rc != SP2B_OK) return rc;
      if (core_d && cs) {
        long long src = 0;
        for (size_t q = 0; q < t_refined.size(); ++q) {
          const int p = t_refined[q];
          long long dst = 0;
          for (int r = 0; r < p; ++r) dst += (long long)lls[r] * (hp[r + 1] - hp[r]);
          const long long m = (long long)lls[p] * (hp[p + 1] - hp[p]);
          SP2B_CUDA_TRY(cudaMemcpyAsync(rho_core + dst, rcore + src, m * sizeof(double),
                                        cudaMemcpyDeviceToHost, st));
          src += m;
        }
        SP2B_CUDA_TRY(cudaStreamSynchronize(st));
      }
      core_out_done = cs != nullptr;
    }
  }

  // ---- outputs ----
  if (vv) {
    for (int k = 0; k < maxiter; ++k) vvh[k] = std::sqrt(vvh[k]);  // prg_fnormGraph
    std::memcpy(vv, vvh.data(), maxiter * sizeof(double));
  }
  if (!dev) {
    if (rho_core && !core_out_done)
      SP2B_CUDA_TRY(cudaMemcpy(rho_core, b.core, coff * sizeof(double), cudaMemcpyDeviceToHost));
    if (rho_dense)
      SP2B_CUDA_TRY(cudaMemcpy(rho_dense, b.dense, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return SP2B_OK;
}

extern "C" int sp2b_last_subgraph_refined(int* count, int* parts, int max_parts, double* idem,
                                          int nparts) {
  if (count) *count = (int)t_refined.size();
  if (parts)
    for (int q = 0; q < std::min(max_parts, (int)t_refined.size()); ++q) parts[q] = t_refined[q];
  if (idem)
    for (int p = 0; p < nparts; ++p) idem[p] = p < (int)t_idem.size() ? t_idem[p] : 0.0;
  return SP2B_OK;
}

extern "C" int sp2b_place_core_rows(long long n, int nparts, const long long* halo_ptr,
                                    const int* halo_idx, const int* llsize,
                                    const long long* src_off, const double* src, double* rho,
                                    void* stream) {
  if (n <= 0 || nparts < 0 || (nparts > 0 && (!halo_ptr || !halo_idx || !llsize || !src_off ||
                                              !src || !rho))) {
    set_last_error("sp2b_place_core_rows: bad argument");
    return SP2B_BAD_ARG;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    set_last_error("no CUDA device available");
    return SP2B_NO_DEVICE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  SP2B_CUDA_TRY(launch_place_core(halo_ptr, halo_idx, llsize, src_off, nparts, src, rho, n, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  return SP2B_OK;
}
