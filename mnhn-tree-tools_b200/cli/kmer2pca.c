/*
 * kmer2pca <kmer file> <projections out> <eigenvalues out> <dimensions> <n_threads>
 *
 * Drop-in for the reference tool (kmer2pca.c:484-597): principal components
 * of a k-mer table (fasta2kmer's output: a label, then the counts, per line).
 * The eigenvalue file gets every eigenvalue of the covariance matrix in
 * ascending order, one "%lf" per line; the projection file gets, per sample,
 * its raw counts projected onto the eigenvectors of the `dimensions` largest
 * eigenvalues, "%lf" tab separated.  Covariance, projections and the
 * reduction and bisection of the eigen-decomposition run on the GPU through
 * libswgpu (the table is uploaded once); n_threads is accepted and ignored.
 * Exits 1 on a missing argument, a file that cannot be opened or read,
 * dimensions outside 1 .. n_features, or a GPU error (the reference reads past
 * its arguments or arrays there).
 */
#define _POSIX_C_SOURCE 200809L
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include "mnhn_dropin.h"
#include "swgpu.h"

static int failed(const char* what, swe_ctx* ctx, int st) {
  printf("%s failed: %s %s\n", what, swe_strerror(st), ctx ? swe_last_error(ctx) : "");
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 6) {
    printf("Arguments are: \n"
           " [FILE-in ] kmer file to apply PCA on \n"
           " [FILE-out] file to write kmers projected onto"
           "principal components to\n"
           " [FILE-out] Eigenvalue Spectrum of the PCA \n"
           " [int] dimensions - how many principal components to project"
           "onto \n"
           " [int] number of threads to use for this computation\n");
    return 1;
  }
  size_t dimensions = 0, n_threads = 1;
  sscanf(argv[4], "%zu", &dimensions);
  sscanf(argv[5], "%zu", &n_threads);
  int infile = open(argv[1], O_RDONLY);
  if (infile < 0) {
    printf("Failed to open input file! \n");
    return 1;
  }
  data_shape shape = shape_from_kmer_file(infile);
  const size_t n = shape.n_samples, nf = shape.n_features;
  if (dimensions < 1 || dimensions > nf || n < 1) {
    printf("dimensions must lie in 1 .. %zu (features) and the table must hold samples\n", nf);
    return 1;
  }
  double* data = malloc(sizeof(double) * nf * n);
  FILE* infilep = fdopen(infile, "r");
  if (!data || !infilep || swe_read_feature_table(infilep, shape, data) != 0) {
    printf("Could not read the table in %s\n", argv[1]);
    return 1;
  }
  printf("Read in data complete: shape: features %lu samples %lu\n", (unsigned long)nf, (unsigned long)n);

  swe_ctx* ctx = NULL;
  swe_opts opts = {0};
  const char* dev = getenv("SWGPU_DEVICE");
  opts.device = dev ? atoi(dev) : 0;
  int st = swe_create(&ctx, &opts);
  if (st) return failed("swe_create", NULL, st);
  double* cov = malloc(sizeof(double) * nf * nf);
  double* eigenvalues = malloc(sizeof(double) * nf);
  double* vectors = malloc(sizeof(double) * nf * dimensions);
  double* projections = malloc(sizeof(double) * n * dimensions);
  if (!cov || !eigenvalues || !vectors || !projections) return failed("allocation", NULL, SWE_ERR_OOM);
  st = swe_pca_covariance(ctx, data, (int64_t)n, (int64_t)nf, cov, NULL);
  if (st) return failed("covariance", ctx, st);
  printf("Means complete \n");
  printf("Covariance complete\n");
  st = swe_pca_eigen_gpu(ctx, cov, (int64_t)nf, (int64_t)dimensions, eigenvalues, vectors);
  if (st) return failed("eigen-decomposition", ctx, st);
  printf("Eigenspace obtained\n");
  st = swe_pca_project(ctx, NULL, (int64_t)n, (int64_t)nf, vectors, (int64_t)dimensions, projections, NULL);
  if (st) return failed("projection", ctx, st);
  swe_destroy(ctx);
  free(cov);
  free(vectors);
  free(data);

  FILE* proj_file = fopen(argv[2], "w");
  FILE* eig_file = fopen(argv[3], "w");
  if (!proj_file || !eig_file) {
    printf("Could not open the output files\n");
    return 1;
  }
  for (size_t i = 0; i < nf; i++) fprintf(eig_file, "%lf\n", eigenvalues[i]);
  for (size_t j = 0; j < n; j++) {
    for (size_t i = 0; i + 1 < dimensions; i++) fprintf(proj_file, "%lf\t", projections[j * dimensions + i]);
    fprintf(proj_file, "%lf\n", projections[j * dimensions + dimensions - 1]);
  }
  free(eigenvalues);
  free(projections);
  fclose(infilep);
  fclose(proj_file);
  fclose(eig_file);
  return 0;
}
