// Host-side logic of the graph-partitioned SP2 path: branch sequence from a gap
// estimate, gap estimate from a recorded sequence, equal partitions, core+halo
// index lists.  Pure C++; no GPU.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/sp2b.h"

extern "C" {

// prg_sp2sequence, src/prg_homolumo_mod.F90:97-147.
int sp2b_sp2sequence(int* pp, int* imax, double mineval, double maxeval, double ehomo,
                     double elumo, double errlimit, int ppmax) {
  if (!pp || !imax || ppmax < 1 || !(maxeval - mineval > 0.0)) return SP2B_BAD_ARG;
  double eh = (maxeval - ehomo) / (maxeval - mineval);
  double el = (maxeval - elumo) / (maxeval - mineval);
  double error = 1.0;
  int it = 0;
  const int cap = ppmax < 100 ? ppmax : 100;  // the reference stops at 100 (:139)
  while (error > errlimit) {
    it += 1;
    // parenthesisation as in the reference (:126-129)
    if ((std::fabs(1.0 - eh * eh) + std::fabs(el * el)) <
        (std::fabs(1.0 - (2.0 * eh - eh * eh) + std::fabs(2.0 * el - el * el))))
      pp[it - 1] = 1;
    else
      pp[it - 1] = 0;
    const double sgm = 1.0 - 2.0 * pp[it - 1];
    eh = eh + sgm * (eh - eh * eh);
    el = el + sgm * (el - el * el);
    error = std::fabs(1.0 - eh) + std::fabs(el);
    if (it >= cap) error = 0.0;
  }
  *imax = it;
  return SP2B_OK;
}

// prg_homolumogap, src/prg_homolumo_mod.F90:22-89.  imax is the 1-based count.
int sp2b_homolumogap(const double* vv, int imax, const int* pp, double mineval, double maxeval,
                     double* ehomo, double* elumo, double* egap) {
  if (!vv || !pp || imax < 1 || !ehomo || !elumo || !egap) return SP2B_BAD_ARG;
  double x_a = 0.0, x_b = 1.0;
  int i = imax;
  while (i >= 1 && vv[i - 1] <= 0.0) i -= 1;
  double hgamma = 6.0 - 4.0 * std::sqrt(2.0);
  hgamma = hgamma * (1.0 - hgamma);
  while (i >= 1 && vv[i - 1] < hgamma) {
    const double precomp = std::sqrt(1.0 - 4.0 * vv[i - 1]);
    double y_a = 0.5 * (1.0 + precomp);
    double y_b = 0.5 * (1.0 - precomp);
    for (int j = i - 1; j >= 1; --j) {
      if (pp[j - 1] > 0) {
        y_a = std::sqrt(y_a);
        y_b = std::sqrt(y_b);
      } else {
        y_a = 1.0 - std::sqrt(1.0 - y_a);
        y_b = 1.0 - std::sqrt(1.0 - y_b);
      }
    }
    x_a = x_a > y_a ? x_a : y_a;
    x_b = x_b < y_b ? x_b : y_b;
    i -= 1;
  }
  *ehomo = maxeval - x_a * (maxeval - mineval);
  *elumo = maxeval - x_b * (maxeval - mineval);
  *egap = *elumo - *ehomo;
  return SP2B_OK;
}

// prg_equalPartition, src/prg_graph_mod.F90:359-399.
int sp2b_equal_partition(int nodes_per_part, int nnodes, int* nparts, int* part_ptr,
                         int* nodes) {
  if (nodes_per_part < 1 || nnodes < 1 || !nparts) return SP2B_BAD_ARG;
  int np;
  if (nnodes <= nodes_per_part)
    np = 1;
  else
    np = (int)std::ceil((float)nnodes / (float)nodes_per_part);
  *nparts = np;
  if (!part_ptr) return SP2B_OK;
  int off = 0;
  for (int i = 1; i <= np; ++i) {
    int psize;
    if (i * nodes_per_part <= nnodes)
      psize = nodes_per_part;
    else
      psize = nnodes - nodes_per_part * (i - 1);
    part_ptr[i - 1] = off;
    if (nodes)
      for (int j = 0; j < psize; ++j) nodes[off + j] = (i - 1) * nodes_per_part + j;
    off += psize;
  }
  part_ptr[np] = off;
  return SP2B_OK;
}

// Core+halo index lists (bml_matrix2submatrix_index as called at
// src/prg_subgraphloop_mod.F90:60-63).  Core nodes first in part order, then nodes
// reached from the core through the graph, then through H, then (double jump) one
// more sweep over the graph rows of every node collected so far.
int sp2b_subgraph_halos(int n, const long long* g_row_ptr, const int* g_col,
                        const long long* h_row_ptr, const int* h_col, int nparts,
                        const int* part_ptr, const int* part_nodes, int double_jump,
                        long long* halo_ptr, int* halo_idx, long long halo_cap,
                        long long* halo_needed, int* lsize, int* llsize) {
  if (n < 1 || !g_row_ptr || !g_col || nparts < 1 || !part_ptr || !part_nodes || !halo_ptr)
    return SP2B_BAD_ARG;
  std::vector<int> mark(n, -1);
  std::vector<int> idx;
  idx.reserve(1024);
  long long off = 0;
  bool overflow = false;
  for (int p = 0; p < nparts; ++p) {
    idx.clear();
    const int a = part_ptr[p], b = part_ptr[p + 1];
    for (int q = a; q < b; ++q) {
      const int v = part_nodes[q];
      if (v < 0 || v >= n) return SP2B_BAD_ARG;
      if (mark[v] != p) {
        mark[v] = p;
        idx.push_back(v);
      }
    }
    const int ncore = (int)idx.size();
    auto sweep = [&](const long long* rp, const int* col, int upto) {
      for (int q = 0; q < upto; ++q) {
        const int v = idx[q];
        for (long long e = rp[v]; e < rp[v + 1]; ++e) {
          const int k = col[e];
          if (k >= 0 && k < n && mark[k] != p) {
            mark[k] = p;
            idx.push_back(k);
          }
        }
      }
    };
    sweep(g_row_ptr, g_col, ncore);
    if (h_row_ptr && h_col) sweep(h_row_ptr, h_col, ncore);
    if (double_jump) sweep(g_row_ptr, g_col, (int)idx.size());
    halo_ptr[p] = off;
    if (halo_idx && off + (long long)idx.size() <= halo_cap)
      std::memcpy(halo_idx + off, idx.data(), idx.size() * sizeof(int));
    else
      overflow = true;
    if (lsize) lsize[p] = (int)idx.size();
    if (llsize) llsize[p] = ncore;
    off += (long long)idx.size();
  }
  halo_ptr[nparts] = off;
  if (halo_needed) *halo_needed = off;
  return overflow ? SP2B_BAD_ARG : SP2B_OK;
}

}  // extern "C"
