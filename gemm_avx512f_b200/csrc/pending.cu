// pending.cu -- entry points whose kernels are not built yet report
// B2_ERR_UNSUPPORTED instead of computing anything.
#include "b2_methods.cuh"
extern "C" {
void dtrsm_(const char *, const char *, const char *, const char *, const int *, const int *,
            const double *, const double *, const int *, double *, const int *) {}
void zgemm3m_(const char *, const char *, const int *, const int *, const int *, const double *,
              const double *, const int *, const double *, const int *, const double *, double *,
              const int *) {}
void cgemm3m_(const char *, const char *, const int *, const int *, const int *, const float *,
              const float *, const int *, const float *, const int *, const float *, float *,
              const int *) {}
int b2_dtrsm(char, char, char, char, int, int, double, const double *, int, double *, int, int,
             int, void *) { return B2_ERR_UNSUPPORTED; }
int b2_zgemm3m(char, char, int, int, int, const double *, const double *, int, const double *,
               int, const double *, double *, int, void *) { return B2_ERR_UNSUPPORTED; }
int b2_cgemm3m(char, char, int, int, int, const float *, const float *, int, const float *, int,
               const float *, float *, int, void *) { return B2_ERR_UNSUPPORTED; }
}
