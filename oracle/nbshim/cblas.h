// CBLAS prototypes for the reference's BLAS calls, resolved at link time
// against an OpenBLAS that exports unprefixed CBLAS symbols.  Oracle-only.
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;
void cblas_sgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, int, int, int,
                 float, const float*, int, const float*, int, float, float*, int);
void cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, int, int, int,
                 double, const double*, int, const double*, int, double, double*, int);
void cblas_ssyrk(enum CBLAS_ORDER, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, int, int,
                 float, const float*, int, float, float*, int);
void cblas_dsyrk(enum CBLAS_ORDER, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, int, int,
                 double, const double*, int, double, double*, int);
void cblas_saxpy(int, float, const float*, int, float*, int);
void cblas_daxpy(int, double, const double*, int, double*, int);
void cblas_sscal(int, float, float*, int);
void cblas_dscal(int, double, double*, int);
float cblas_sdot(int, const float*, int, const float*, int);
double cblas_ddot(int, const double*, int, const double*, int);
void cblas_sgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int, int, float, const float*, int,
                 const float*, int, float, float*, int);
void cblas_dgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int, int, double, const double*, int,
                 const double*, int, double, double*, int);
char* openblas_get_config(void);
void openblas_set_num_threads(int);
#ifdef __cplusplus
}
#endif
