/* A plain C client of the C-ABI (C99, no CUDA headers): reads a FEAT3 binary CSR file and a
 * FEAT3 binary vector, writes them back in FEAT3's formats and checks the round trip. The I/O
 * entry points are host code, so this runs without a GPU.
 *   io_client <matrix.csr> <vector.dv> <out_dir> */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "feat3_b200.h"

static int same_file(const char* a, const char* b) {
  FILE* fa = fopen(a, "rb");
  FILE* fb = fopen(b, "rb");
  int same = fa && fb;
  while (same) {
    int ca = fgetc(fa), cb = fgetc(fb);
    if (ca != cb) same = 0;
    if (ca == EOF || cb == EOF) break;
  }
  if (fa) fclose(fa);
  if (fb) fclose(fb);
  return same;
}

int main(int argc, char** argv) {
  if (argc != 4) return 2;
  char path[4096];
  fb_csr_host m;
  int rc = fb_io_csr_read(argv[1], FB_FILE_CSR, &m);
  if (rc != FB_OK) { fprintf(stderr, "read matrix: %d\n", rc); return 1; }
  printf("matrix %llu x %llu, %llu entries, row_ptr[rows] = %llu\n", (unsigned long long)m.rows,
         (unsigned long long)m.cols, (unsigned long long)m.nnz, (unsigned long long)m.row_ptr[m.rows]);
  snprintf(path, sizeof(path), "%s/m.csr", argv[3]);
  if ((rc = fb_io_csr_write(path, FB_FILE_BINARY, &m, 0)) != FB_OK) { fprintf(stderr, "write: %d\n", rc); return 1; }
  if (!same_file(path, argv[1])) { fprintf(stderr, "binary round trip differs\n"); return 1; }
  uint64_t size = 0;
  if (fb_io_csr_serialised_size(&m, &size) != FB_OK) return 1;
  void* buf = malloc(size);
  if (!buf || fb_io_csr_serialise(&m, buf, size) != FB_OK) return 1;
  if (fb_io_csr_serialise(&m, buf, size - 1) != FB_ERR_TOO_LARGE) { fprintf(stderr, "capacity not checked\n"); return 1; }
  fb_csr_host back;
  if (fb_io_csr_deserialise(buf, size, &back) != FB_OK || back.nnz != m.nnz ||
      memcmp(back.val, m.val, m.nnz * sizeof(double)) != 0 ||
      memcmp(back.col_ind, m.col_ind, m.nnz * sizeof(uint64_t)) != 0) {
    fprintf(stderr, "in-memory round trip differs\n");
    return 1;
  }
  fb_io_csr_release(&back);
  free(buf);
  snprintf(path, sizeof(path), "%s/m.mtx", argv[3]);
  if (fb_io_csr_write(path, FB_FILE_MTX, &m, 1) != FB_OK) return 1;
  fb_csr_host sym;
  if (fb_io_csr_read(path, FB_FILE_MTX, &sym) != FB_OK || sym.nnz != m.nnz) { fprintf(stderr, "symmetric mtx\n"); return 1; }
  fb_io_csr_release(&sym);
  fb_io_csr_release(&m);
  uint64_t n = 0;
  double* v = NULL;
  if ((rc = fb_io_vector_read(argv[2], FB_FILE_DV, &n, &v)) != FB_OK) { fprintf(stderr, "read vector: %d\n", rc); return 1; }
  snprintf(path, sizeof(path), "%s/v.dv", argv[3]);
  if (fb_io_vector_write(path, FB_FILE_DV, v, n) != FB_OK || !same_file(path, argv[2])) return 1;
  printf("vector %llu values\n", (unsigned long long)n);
  fb_io_free(v);
  if (fb_io_csr_read("/nonexistent/file.csr", FB_FILE_CSR, &m) != FB_ERR_IO) return 1;
  printf("%s: ok\n", fb_version());
  return 0;
}
