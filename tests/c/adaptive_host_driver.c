/*
 * Test driver for the adaptive_dbscan function-pointer seam (dbscan.h:72-81)
 * without a GPU: the dbscanner below thresholds a distance matrix read from a
 * file (written by the oracle) and runs libswgpu's DBSCAN replay on it;
 * libswgpu's adaptive_dbscan drives it and writes the log and split sets.
 *
 *   adaptive_host_driver <fasta> <matrix.swd> <eps_start> <eps_inc> <minpts> <prefix>
 *
 * The matrix file is "SWD1", uint32 n, uint32 element size (2 or 4), then n*n
 * row-major little-endian distances.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mnhn_dropin.h"
#include "swgpu.h"

static uint32_t* g_D;
static int g_n;

static split_set matrix_dbscanner(dataset ds, float eps, int minpts) {
  split_set out = {0, NULL};
  int n = ds.n_values, wpr = (n + 63) / 64;
  uint64_t* bits = (uint64_t*)calloc((size_t)n * wpr + 1, 8);
  int* counts = (int*)calloc((size_t)n + 1, sizeof(int));
  if (eps == -1) eps = 0.015f;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++)
      if ((float)g_D[(size_t)i * g_n + k] <= eps) {
        bits[(size_t)i * wpr + k / 64] |= 1ull << (k % 64);
        counts[i]++;
      }
  swe_dbscan_bitmap(n, bits, wpr, counts, minpts, &out);
  free(bits);
  free(counts);
  return out;
}

int main(int argc, char** argv) {
  if (argc < 7) return 2;
  FILE* f = fopen(argv[1], "r");
  if (!f) return 2;
  dataset ds = dataset_from_fasta(f);
  fclose(f);
  FILE* m = fopen(argv[2], "rb");
  char magic[4];
  uint32_t n, es;
  if (!m || fread(magic, 1, 4, m) != 4 || memcmp(magic, "SWD1", 4) || fread(&n, 4, 1, m) != 1 ||
      fread(&es, 4, 1, m) != 1 || (int)n != ds.n_values)
    return 3;
  g_n = (int)n;
  g_D = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n * n + 4);
  for (size_t k = 0; k < (size_t)n * n; k++) {
    uint32_t v = 0;
    if (fread(&v, es, 1, m) != 1) return 3;
    g_D[k] = v;
  }
  fclose(m);
  printf("Dataset read!\n");
  adaptive_dbscan(matrix_dbscanner, ds, strtof(argv[3], NULL), strtof(argv[4], NULL), atoi(argv[5]), argv[6], 1);
  fflush(stdout);
  return swgpu_last_dropin_status() ? 1 : 0;
}
