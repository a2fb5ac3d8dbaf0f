/*
 * Test infrastructure only (oracle). The reference calls Fortran BLAS/LAPACK
 * symbols (dgemm_, dtrsm_, dpotrf_, ...), normally from MKL. MKL is not in
 * this image, so these forwarders route each one to the OpenBLAS build that
 * ships with scipy, whose symbols carry a scipy_ prefix. Arguments pass through
 * unchanged, by reference, as in the Fortran ABI (character arguments are
 * single letters; the hidden length arguments are not needed by OpenBLAS).
 */
typedef int I;
typedef double D;
typedef struct { double re, im; } Z;
typedef struct { float re, im; } C;

#define P const

extern void scipy_dscal_(P I*, P D*, D*, P I*);
extern void scipy_zscal_(P I*, P Z*, Z*, P I*);
extern void scipy_dcopy_(P I*, P D*, P I*, D*, P I*);
extern void scipy_zcopy_(P I*, P Z*, P I*, Z*, P I*);
extern void scipy_dgemm_(P char*, P char*, P I*, P I*, P I*, P D*, P D*, P I*, P D*, P I*, P D*,
                         D*, P I*);
extern void scipy_zgemm_(P char*, P char*, P I*, P I*, P I*, P Z*, P Z*, P I*, P Z*, P I*, P Z*,
                         Z*, P I*);
extern void scipy_dtrsm_(P char*, P char*, P char*, P char*, P I*, P I*, P D*, P D*, P I*, D*,
                         P I*);
extern void scipy_dlacpy_(P char*, P I*, P I*, P D*, P I*, D*, P I*);
extern void scipy_zlacpy_(P char*, P I*, P I*, P Z*, P I*, Z*, P I*);
extern void scipy_spotrf_(P char*, P I*, float*, P I*, I*);
extern void scipy_dpotrf_(P char*, P I*, D*, P I*, I*);
extern void scipy_cpotrf_(P char*, P I*, C*, P I*, I*);
extern void scipy_zpotrf_(P char*, P I*, Z*, P I*, I*);
extern void scipy_dgesvd_(P char*, P char*, P I*, P I*, D*, P I*, D*, D*, P I*, D*, P I*, D*,
                          P I*, I*);

void dscal_(P I* n, P D* a, D* x, P I* ix) { scipy_dscal_(n, a, x, ix); }
void zscal_(P I* n, P Z* a, Z* x, P I* ix) { scipy_zscal_(n, a, x, ix); }
void dcopy_(P I* n, P D* x, P I* ix, D* y, P I* iy) { scipy_dcopy_(n, x, ix, y, iy); }
void zcopy_(P I* n, P Z* x, P I* ix, Z* y, P I* iy) { scipy_zcopy_(n, x, ix, y, iy); }
void dgemm_(P char* ta, P char* tb, P I* m, P I* n, P I* k, P D* al, P D* a, P I* lda, P D* b,
            P I* ldb, P D* be, D* c, P I* ldc) {
  scipy_dgemm_(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc);
}
void zgemm_(P char* ta, P char* tb, P I* m, P I* n, P I* k, P Z* al, P Z* a, P I* lda, P Z* b,
            P I* ldb, P Z* be, Z* c, P I* ldc) {
  scipy_zgemm_(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc);
}
void dtrsm_(P char* s, P char* u, P char* t, P char* d, P I* m, P I* n, P D* al, P D* a, P I* lda,
            D* b, P I* ldb) {
  scipy_dtrsm_(s, u, t, d, m, n, al, a, lda, b, ldb);
}
void dlacpy_(P char* u, P I* m, P I* n, P D* a, P I* lda, D* b, P I* ldb) {
  scipy_dlacpy_(u, m, n, a, lda, b, ldb);
}
void zlacpy_(P char* u, P I* m, P I* n, P Z* a, P I* lda, Z* b, P I* ldb) {
  scipy_zlacpy_(u, m, n, a, lda, b, ldb);
}
void spotrf_(P char* u, P I* n, float* a, P I* lda, I* info) { scipy_spotrf_(u, n, a, lda, info); }
void dpotrf_(P char* u, P I* n, D* a, P I* lda, I* info) { scipy_dpotrf_(u, n, a, lda, info); }
void cpotrf_(P char* u, P I* n, C* a, P I* lda, I* info) { scipy_cpotrf_(u, n, a, lda, info); }
void zpotrf_(P char* u, P I* n, Z* a, P I* lda, I* info) { scipy_zpotrf_(u, n, a, lda, info); }
void dgesvd_(P char* ju, P char* jv, P I* m, P I* n, D* a, P I* lda, D* s, D* u, P I* ldu, D* vt,
             P I* ldvt, D* w, P I* lw, I* info) {
  scipy_dgesvd_(ju, jv, m, n, a, lda, s, u, ldu, vt, ldvt, w, lw, info);
}
