/*
 * fftw_shim.c -- project-written implementation of the FFTW3 entry points the
 * reference's SOFT sources (phaser_core/lib/SOFT) and its phaser_core glue
 * call.  It lets oracle/Makefile compile those sources, unmodified, where they
 * lie in the reference tree.  Not FFTW code: every transform is computed from
 * its definition with the FP64 Stockham FFT of fft64.h.
 * TEST INFRASTRUCTURE ONLY.
 */
#include "fftw3/fftw3.h"

#include <stdint.h>

#include "fft64.h"

#ifdef _OPENMP
#include <omp.h>
#endif

enum { P_R2R = 1, P_SPLIT = 2, P_MANY = 3, P_R2C3 = 4, P_C2R3 = 5 };

struct fftw_plan_s {
  int kind;
  int sign;
  /* r2r */
  int n;
  double* rin;
  double* rout;
  /* split */
  fftw_iodim dim, hdim;
  double *ri, *ii, *ro, *io;
  /* many */
  int rank, nn[3], inem[3], onem[3], howmany, istride, idist, ostride, odist;
  fftw_complex *cin, *cout;
  /* 3d */
  int n0, n1, n2;
  /* cached 1-D plan for r2r / split */
  orc_fft_plan fp;
  int has_fp;
};

static int g_threads = 1;

void* fftw_malloc(size_t n) {
  void* p = NULL;
  if (posix_memalign(&p, 64, n ? n : 16) != 0) return NULL;
  return p;
}

void fftw_free(void* p) { free(p); }

int fftw_init_threads(void) { return 1; }

void fftw_plan_with_nthreads(int n) { g_threads = n > 0 ? n : 1; }

void fftw_cleanup(void) {}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  if (p->has_fp) plan_free(&p->fp);
  free(p);
}

static fftw_plan new_plan(int kind) {
  fftw_plan p = (fftw_plan)calloc(1, sizeof(struct fftw_plan_s));
  p->kind = kind;
  return p;
}

fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind,
                           unsigned flags) {
  (void)flags;
  if (kind != FFTW_REDFT10) return NULL;
  fftw_plan p = new_plan(P_R2R);
  p->n = n;
  plan_init(&p->fp, n);
  p->has_fp = 1;
  p->rin = in;
  p->rout = out;
  return p;
}

fftw_plan fftw_plan_guru_split_dft(int rank, const fftw_iodim* dims,
                                   int howmany_rank,
                                   const fftw_iodim* howmany_dims, double* ri,
                                   double* ii, double* ro, double* io,
                                   unsigned flags) {
  (void)flags;
  if (rank != 1 || howmany_rank != 1) return NULL;
  fftw_plan p = new_plan(P_SPLIT);
  p->dim = dims[0];
  plan_init(&p->fp, dims[0].n);
  p->has_fp = 1;
  p->hdim = howmany_dims[0];
  p->ri = ri;
  p->ii = ii;
  p->ro = ro;
  p->io = io;
  return p;
}

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
                             fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed,
                             int ostride, int odist, int sign, unsigned flags) {
  (void)flags;
  if (rank < 1 || rank > 3) return NULL;
  fftw_plan p = new_plan(P_MANY);
  p->rank = rank;
  for (int d = 0; d < rank; ++d) {
    p->nn[d] = n[d];
    p->inem[d] = inembed ? inembed[d] : n[d];
    p->onem[d] = onembed ? onembed[d] : n[d];
  }
  p->howmany = howmany;
  p->cin = in;
  p->cout = out;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->sign = sign;
  return p;
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in,
                               fftw_complex* out, unsigned flags) {
  (void)flags;
  fftw_plan p = new_plan(P_R2C3);
  p->n0 = n0;
  p->n1 = n1;
  p->n2 = n2;
  p->rin = in;
  p->cout = out;
  return p;
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in,
                               double* out, unsigned flags) {
  (void)flags;
  fftw_plan p = new_plan(P_C2R3);
  p->n0 = n0;
  p->n1 = n1;
  p->n2 = n2;
  p->cin = in;
  p->rout = out;
  return p;
}

void fftw_execute_r2r(const fftw_plan p, double* in, double* out) {
  const orc_fft_plan* fp = &p->fp;
  cplx* v = (cplx*)malloc(sizeof(cplx) * (size_t)p->n);
  cplx* s = (cplx*)malloc(sizeof(cplx) * (size_t)p->n);
  double* tmp = (double*)malloc(sizeof(double) * (size_t)p->n);
  dct2_exec(fp, in, tmp, v, s);
  memcpy(out, tmp, sizeof(double) * (size_t)p->n);
  free(v);
  free(s);
  free(tmp);
}

void fftw_execute_split_dft(const fftw_plan p, double* ri, double* ii,
                            double* ro, double* io) {
  const int n = p->dim.n;
  const orc_fft_plan* fp = &p->fp;
#pragma omp parallel num_threads(g_threads)
  {
    cplx* x = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    cplx* s = (cplx*)malloc(sizeof(cplx) * (size_t)n);
#pragma omp for
    for (int h = 0; h < p->hdim.n; ++h) {
      for (int j = 0; j < n; ++j) {
        x[j].re = ri[(long)h * p->hdim.is + (long)j * p->dim.is];
        x[j].im = ii[(long)h * p->hdim.is + (long)j * p->dim.is];
      }
      fft_exec(fp, x, s, -1);
      for (int k = 0; k < n; ++k) {
        ro[(long)h * p->hdim.os + (long)k * p->dim.os] = x[k].re;
        io[(long)h * p->hdim.os + (long)k * p->dim.os] = x[k].im;
      }
    }
    free(x);
    free(s);
  }
}

/* One rank-r transform of the "many" plan along every dimension. */
static void many_exec(const fftw_plan p) {
  const int r = p->rank;
  long tot = 1;
  for (int d = 0; d < r; ++d) tot *= p->nn[d];
  long istr[3], ostr[3];
  istr[r - 1] = 1;
  ostr[r - 1] = 1;
  for (int d = r - 2; d >= 0; --d) {
    istr[d] = istr[d + 1] * p->inem[d + 1];
    ostr[d] = ostr[d + 1] * p->onem[d + 1];
  }
#pragma omp parallel num_threads(g_threads)
  {
    cplx* buf = (cplx*)malloc(sizeof(cplx) * (size_t)tot);
    int nmax = 1;
    for (int d = 0; d < r; ++d) nmax = p->nn[d] > nmax ? p->nn[d] : nmax;
    cplx* row = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
    cplx* scr = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
    orc_fft_plan fp[3];
    for (int d = 0; d < r; ++d) plan_init(&fp[d], p->nn[d]);
#pragma omp for
    for (int h = 0; h < p->howmany; ++h) {
      /* gather into a dense row-major buffer */
      for (long e = 0; e < tot; ++e) {
        long rem = e, off = 0;
        for (int d = r - 1; d >= 0; --d) {
          off += (rem % p->nn[d]) * istr[d];
          rem /= p->nn[d];
        }
        const double* src = p->cin[(long)h * p->idist + off * p->istride];
        buf[e].re = src[0];
        buf[e].im = src[1];
      }
      long inner = 1;
      for (int d = r - 1; d >= 0; --d) {
        const int nd = p->nn[d];
        if (nd > 1) {
          const long outer = tot / (inner * nd);
          for (long o = 0; o < outer; ++o)
            for (long in = 0; in < inner; ++in) {
              const long base = o * nd * inner + in;
              for (int k = 0; k < nd; ++k) row[k] = buf[base + (long)k * inner];
              fft_exec(&fp[d], row, scr, p->sign);
              for (int k = 0; k < nd; ++k) buf[base + (long)k * inner] = row[k];
            }
        }
        inner *= nd;
      }
      for (long e = 0; e < tot; ++e) {
        long rem = e, off = 0;
        for (int d = r - 1; d >= 0; --d) {
          off += (rem % p->nn[d]) * ostr[d];
          rem /= p->nn[d];
        }
        double* dst = p->cout[(long)h * p->odist + off * p->ostride];
        dst[0] = buf[e].re;
        dst[1] = buf[e].im;
      }
    }
    for (int d = 0; d < r; ++d) plan_free(&fp[d]);
    free(buf);
    free(row);
    free(scr);
  }
}

static void fft3(cplx* a, int n0, int n1, int n2, int sign) {
  orc_fft_plan p0, p1, p2;
  plan_init(&p0, n0);
  plan_init(&p1, n1);
  plan_init(&p2, n2);
  int nmax = n0 > n1 ? n0 : n1;
  if (n2 > nmax) nmax = n2;
#pragma omp parallel num_threads(g_threads)
  {
    cplx* row = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
    cplx* scr = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for
    for (long r = 0; r < (long)n0 * n1; ++r) fft_exec(&p2, a + r * n2, scr, sign);
#pragma omp for
    for (long r = 0; r < (long)n0 * n2; ++r) {
      const long i0 = r / n2, i2 = r % n2;
      for (int i1 = 0; i1 < n1; ++i1) row[i1] = a[(i0 * n1 + i1) * n2 + i2];
      fft_exec(&p1, row, scr, sign);
      for (int i1 = 0; i1 < n1; ++i1) a[(i0 * n1 + i1) * n2 + i2] = row[i1];
    }
#pragma omp for
    for (long r = 0; r < (long)n1 * n2; ++r) {
      for (int i0 = 0; i0 < n0; ++i0) row[i0] = a[(long)i0 * n1 * n2 + r];
      fft_exec(&p0, row, scr, sign);
      for (int i0 = 0; i0 < n0; ++i0) a[(long)i0 * n1 * n2 + r] = row[i0];
    }
    free(row);
    free(scr);
  }
  plan_free(&p0);
  plan_free(&p1);
  plan_free(&p2);
}

static void r2c3_exec(const fftw_plan p) {
  const long n0 = p->n0, n1 = p->n1, n2 = p->n2, h2 = n2 / 2 + 1;
  const long nv = n0 * n1 * n2;
  cplx* a = (cplx*)malloc(sizeof(cplx) * (size_t)nv);
  for (long i = 0; i < nv; ++i) {
    a[i].re = p->rin[i];
    a[i].im = 0.0;
  }
  fft3(a, (int)n0, (int)n1, (int)n2, -1);
  for (long r = 0; r < n0 * n1; ++r)
    for (long k = 0; k < h2; ++k) {
      p->cout[r * h2 + k][0] = a[r * n2 + k].re;
      p->cout[r * h2 + k][1] = a[r * n2 + k].im;
    }
  free(a);
}

/* c2r: complex inverse along the leading axes, then along the last axis the
 * real output of a half-complex row (DC and Nyquist imaginary parts unread). */
static void c2r3_exec(const fftw_plan p) {
  const long n0 = p->n0, n1 = p->n1, n2 = p->n2, h2 = n2 / 2 + 1;
  const long nv = n0 * n1 * n2;
  cplx* a = (cplx*)calloc((size_t)nv, sizeof(cplx));
  for (long r = 0; r < n0 * n1; ++r)
    for (long k = 0; k < h2; ++k) {
      const double w = (k == 0 || (n2 % 2 == 0 && k == n2 / 2)) ? 1.0 : 2.0;
      a[r * n2 + k].re = w * p->cin[r * h2 + k][0];
      a[r * n2 + k].im = w * p->cin[r * h2 + k][1];
    }
  fft3(a, (int)n0, (int)n1, (int)n2, +1);
  for (long i = 0; i < nv; ++i) p->rout[i] = a[i].re;
  free(a);
}

void fftw_execute(const fftw_plan p) {
  switch (p->kind) {
    case P_R2R:
      fftw_execute_r2r(p, p->rin, p->rout);
      break;
    case P_SPLIT:
      fftw_execute_split_dft(p, p->ri, p->ii, p->ro, p->io);
      break;
    case P_MANY:
      many_exec(p);
      break;
    case P_R2C3:
      r2c3_exec(p);
      break;
    case P_C2R3:
      c2r3_exec(p);
      break;
    default:
      break;
  }
}
