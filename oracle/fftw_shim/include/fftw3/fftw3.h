/*
 * Minimal FFTW3-compatible API declarations, written for this project so the
 * reference's vendored SOFT sources (which include <fftw3/fftw3.h>) can be
 * compiled here without FFTW.  Only the entry points SOFT and the phaser_core
 * glue call are declared.  The implementation (fftw_shim.c) computes the
 * transforms from their definitions in FP64.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef PHASER_ORACLE_FFTW3_SHIM_H_
#define PHASER_ORACLE_FFTW3_SHIM_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

typedef struct {
  int n, is, os;
} fftw_iodim;

typedef enum { FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2, FFTW_REDFT00 = 3,
               FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6 } fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);

fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind,
                           unsigned flags);
fftw_plan fftw_plan_guru_split_dft(int rank, const fftw_iodim* dims,
                                   int howmany_rank,
                                   const fftw_iodim* howmany_dims, double* ri,
                                   double* ii, double* ro, double* io,
                                   unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
                             fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed,
                             int ostride, int odist, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in,
                               fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in,
                               double* out, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftw_execute_r2r(const fftw_plan p, double* in, double* out);
void fftw_execute_split_dft(const fftw_plan p, double* ri, double* ii,
                            double* ro, double* io);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);

#ifdef __cplusplus
}
#endif

#endif /* PHASER_ORACLE_FFTW3_SHIM_H_ */
