/* A stand-in for the part of BML's C API that libsp2b resolves at call time
 * (bml_get_N, bml_get_M, bml_get_type, bml_get_precision, bml_get_distribution_mode,
 * bml_export_to_dense, bml_import_from_dense, bml_copy, bml_deallocate,
 * bml_free_memory), over its own matrix struct, with the enum values of BML's
 * bml_types.h.  Test infrastructure: the PROGRESS-named exports must treat these
 * handles as BML matrices, unchanged.  Counters record how they were used. */
#include <stdlib.h>
#include <string.h>

enum { SINGLE_REAL = 1, DOUBLE_REAL = 2 };
enum { ROW_MAJOR = 0, COLUMN_MAJOR = 1 };

typedef struct {
  int type, prec, N, M, distrib;
  void* d;               /* N x N, column-major, float or double */
  int exports, copies_in;
} stub_t;

static int g_live = 0;   /* matrices allocated and not deallocated */

static size_t esz(int prec) { return prec == SINGLE_REAL ? sizeof(float) : sizeof(double); }

stub_t* stub_new(int type, int prec, int n, int m, const double* colmajor) {
  stub_t* a = (stub_t*)calloc(1, sizeof(stub_t));
  a->type = type;
  a->prec = prec;
  a->N = n;
  a->M = m;
  a->d = calloc((size_t)n * n, esz(prec));
  for (size_t i = 0; colmajor && i < (size_t)n * n; ++i) {
    if (prec == SINGLE_REAL) ((float*)a->d)[i] = (float)colmajor[i];
    else ((double*)a->d)[i] = colmajor[i];
  }
  ++g_live;
  return a;
}
void stub_get(const stub_t* a, double* out) {
  for (size_t i = 0; i < (size_t)a->N * a->N; ++i)
    out[i] = a->prec == SINGLE_REAL ? (double)((float*)a->d)[i] : ((double*)a->d)[i];
}
int stub_exports(const stub_t* a) { return a->exports; }
int stub_copies_in(const stub_t* a) { return a->copies_in; }
int stub_live(void) { return g_live; }
void stub_free(stub_t* a) {
  free(a->d);
  free(a);
  --g_live;
}

int bml_get_N(stub_t* a) { return a->N; }
int bml_get_M(stub_t* a) { return a->M; }
int bml_get_type(stub_t* a) { return a->type; }
int bml_get_precision(stub_t* a) { return a->prec; }
int bml_get_distribution_mode(stub_t* a) { return a->distrib; }

void* bml_export_to_dense(stub_t* a, int order) {
  const size_t n = (size_t)a->N, e = esz(a->prec);
  unsigned char* out = (unsigned char*)malloc(n * n * e);
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j) {
      const size_t src = j * n + i;   /* column-major storage */
      const size_t dst = order == COLUMN_MAJOR ? src : i * n + j;
      memcpy(out + dst * e, (unsigned char*)a->d + src * e, e);
    }
  ++a->exports;
  return out;
}

stub_t* bml_import_from_dense(int type, int prec, int order, int n, int m, void* src,
                              double threshold, int distrib) {
  stub_t* a = stub_new(type, prec, n, m, NULL);
  const size_t e = esz(prec);
  a->distrib = distrib;
  for (size_t i = 0; i < (size_t)n; ++i)
    for (size_t j = 0; j < (size_t)n; ++j) {
      const size_t dst = j * (size_t)n + i;
      const size_t s = order == COLUMN_MAJOR ? dst : i * (size_t)n + j;
      memcpy((unsigned char*)a->d + dst * e, (unsigned char*)src + s * e, e);
      double v = prec == SINGLE_REAL ? (double)((float*)a->d)[dst] : ((double*)a->d)[dst];
      if (type != 1 && (v < 0 ? -v : v) < threshold) {   /* sparse types drop small values */
        if (prec == SINGLE_REAL) ((float*)a->d)[dst] = 0.f;
        else ((double*)a->d)[dst] = 0.0;
      }
    }
  return a;
}

void bml_copy(stub_t* a, stub_t* b) {
  memcpy(b->d, a->d, (size_t)a->N * a->N * esz(a->prec));
  ++b->copies_in;
}

void bml_deallocate(stub_t** a) {
  if (a && *a) {
    stub_free(*a);
    *a = NULL;
  }
}

void bml_free_memory(void* p) { free(p); }
