/* Test infrastructure only.  The reference's kmer2pca.c calls LAPACK's dsyev_
 * (kmer2pca.c:18, 126) and its makefile links -llapack (makefile:8, 84-86).
 * This image has no system LAPACK, but scipy ships OpenBLAS, LAPACK included,
 * with its symbols prefixed "scipy_" (32-bit integers, the Fortran calling
 * convention the reference uses).  This forwards the reference's call to it
 * unchanged, so oracle/_ref/kmer2pca is the reference's own code on a real
 * dsyev. */
void scipy_dsyev_(char* jobz, char* uplo, int* n, double* a, int* lda, double* w, double* work, int* lwork,
                  int* info);

void dsyev_(char* jobz, char* uplo, int* n, double* a, int* lda, double* w, double* work, int* lwork, int* info) {
  scipy_dsyev_(jobz, uplo, n, a, lda, w, work, lwork, info);
}
