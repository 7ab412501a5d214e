/*
 * ref_glue.c -- drives the reference's own SOFT sources (compiled unmodified
 * from phaser_core/lib/SOFT by oracle/Makefile) the way phaser_core's classes
 * do, so the reference's CPU path can be run here:
 *
 *   ref_sht                      SphericalCorrelation::initializeAll +
 *                                performSphericalTransforms
 *                                (phaser_core/src/backend/correlation/
 *                                spherical-correlation.cc:122-246)
 *   ref_spherical_correlation    SphericalCorrelationLaplace::
 *                                correlateSampledSignals
 *                                (spherical-correlation-laplace.cc:14-113) and
 *                                SphericalCorrelation::correlate/
 *                                inverseTransform (spherical-correlation.cc:
 *                                248-279)
 *   ref_spatial_correlation      SpatialCorrelation[Laplace]::correlateSignals
 *                                with its N^3-long half-spectrum buffers
 *                                (spatial-correlation.cc:11-161,
 *                                spatial-correlation-laplace.cc:9-89)
 *   ref_register_pair            SphOptRegistration::registerPointCloud with a
 *                                kd-tree nearest-neighbour sampler, the CPU
 *                                baseline of the benchmark.
 *
 * The phaser_core glue itself needs glog/Eigen/PCL, which are absent, so it is
 * restated here in C.  FFTW entry points come from fftw_shim.c.
 * TEST INFRASTRUCTURE ONLY.
 */
#include <fftw3/fftw3.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "soft/makeweights.h"
#include "soft/s2_cospmls.h"
#include "soft/s2_semi_memo.h"
#include "soft/so3_correlate_fftw.h"
#include "soft/soft_fftw.h"

/* oracle helpers (phaser_oracle.c) */
void orc_fftshift(double* re_im, size_t n);
void orc_ifftshift(double* re_im, size_t n);
void orc_fuse_channels_literal(const double* channels, int C, uint32_t n,
                               int levels, float div, double* out);
void orc_dh_grid(int bw, float* xyz);
void orc_project(const float* pts, size_t stride, size_t P, float* out_xyz,
                 double* range);
void orc_discretize(const float* xyzi, size_t P, const float* refl,
                    const float* amb, int N, int lo, int hi, double* out);
void orc_bin_to_zyz(uint32_t loc, uint32_t bw, double* zyz);
void orc_zyz_to_quat(const double* zyz, double* q);
void orc_quat_to_xyz(const double* q, double* xyz);
void orc_rotation_xyz(float a, float b, float c, float* T);
void orc_transform(float* xyzi, size_t P, const float* T);
uint64_t orc_argmax(const double* v, uint64_t n);
void orc_ind2sub(uint32_t lin, uint32_t rows, uint32_t cols, uint32_t* xyz);
double orc_translation_from_index(double index, uint32_t n_voxels, int lo,
                                  int hi);

/* ------------------------------------------------------------------------ */
/* Spherical correlation object (state of SphericalCorrelation).            */
/* ------------------------------------------------------------------------ */
typedef struct {
  int bw, bw_out;
  fftw_plan dct_plan, fft_plan, inverse_so3;
  fftw_complex *workspace1, *workspace2, *workspace2_out, *so3_sig, *so3_coef;
  double *workspace3, *workspace3_out, *weights;
  double *sig_coef[2], *pat_coef[2], *tmp_coef[2];
  double *tablespace;
  double** table;
} sph_state;

static void sph_init(sph_state* s, int bw, int bw_out) {
  memset(s, 0, sizeof(*s));
  s->bw = bw;
  s->bw_out = bw_out;
  const int n = 2 * bw, n_out = 2 * bw_out;
  const long so3_bw = 8L * bw_out * bw_out * bw_out;
  s->workspace1 = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * so3_bw);
  s->workspace2 = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * (14L * bw * bw + 48L * bw));
  s->workspace3 = (double*)malloc(sizeof(double) * (12L * n + (long)n * bw));
  s->workspace2_out = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * (14L * bw_out * bw_out + 48L * bw_out));
  s->workspace3_out = (double*)malloc(sizeof(double) * (12L * n_out + (long)n_out * bw_out));
  s->weights = (double*)malloc(sizeof(double) * 4 * bw);
  for (int i = 0; i < 2; ++i) {
    s->sig_coef[i] = (double*)malloc(sizeof(double) * bw * bw);
    s->pat_coef[i] = (double*)malloc(sizeof(double) * bw * bw);
    s->tmp_coef[i] = (double*)malloc(sizeof(double) * n * n);
  }
  s->so3_sig = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * so3_bw);
  s->so3_coef = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * ((4L * bw_out * bw_out * bw_out - bw_out) / 3));
  s->tablespace = (double*)malloc(sizeof(double) * (Reduced_Naive_TableSize(bw, bw) + Reduced_SpharmonicTableSize(bw, bw)));
  s->dct_plan = fftw_plan_r2r_1d(n, s->weights, s->workspace3, FFTW_REDFT10, FFTW_ESTIMATE);
  fftw_iodim dims = {n, 1, n};
  fftw_iodim hdims = {n, n, 1};
  s->fft_plan = fftw_plan_guru_split_dft(1, &dims, 1, &hdims, s->tmp_coef[0], s->tmp_coef[1],
                                         (double*)s->workspace2, (double*)s->workspace2 + (n * n),
                                         FFTW_ESTIMATE);
  int na[2] = {1, n_out};
  int inembed[2] = {n_out, n_out * n_out};
  int onembed[2] = {n_out, n_out * n_out};
  s->inverse_so3 = fftw_plan_many_dft(2, na, n_out * n_out, s->workspace1, inembed, 1, n_out,
                                      s->so3_sig, onembed, 1, n_out, FFTW_FORWARD, FFTW_ESTIMATE);
  s->table = SemiNaive_Naive_Pml_Table(bw, bw, s->tablespace, (double*)s->workspace2);
  makeweights(bw, s->weights);
}

static void sph_free(sph_state* s) {
  free(s->workspace3);
  free(s->weights);
  free(s->table);
  free(s->tablespace);
  fftw_destroy_plan(s->inverse_so3);
  fftw_destroy_plan(s->fft_plan);
  fftw_destroy_plan(s->dct_plan);
  fftw_free(s->workspace1);
  fftw_free(s->workspace2);
  fftw_free(s->workspace2_out);
  free(s->workspace3_out);
  fftw_free(s->so3_sig);
  fftw_free(s->so3_coef);
  for (int i = 0; i < 2; ++i) {
    free(s->pat_coef[i]);
    free(s->sig_coef[i]);
    free(s->tmp_coef[i]);
  }
}

static void sph_transform_pair(sph_state* s, const double* f1, const double* f2) {
  const int n = 2 * s->bw;
  for (int i = 0; i < n * n; ++i) {
    s->tmp_coef[0][i] = f1[i];
    s->tmp_coef[1][i] = 0.0;
  }
  FST_semi_memo(s->tmp_coef[0], s->tmp_coef[1], s->sig_coef[0], s->sig_coef[1], s->bw, s->table,
                (double*)s->workspace2, 1, s->bw, &s->dct_plan, &s->fft_plan, s->weights);
  for (int i = 0; i < n * n; ++i) {
    s->tmp_coef[0][i] = f2[i];
    s->tmp_coef[1][i] = 0.0;
  }
  FST_semi_memo(s->tmp_coef[0], s->tmp_coef[1], s->pat_coef[0], s->pat_coef[1], s->bw, s->table,
                (double*)s->workspace2, 1, s->bw, &s->dct_plan, &s->fft_plan, s->weights);
}

static void sph_correlate_inverse(sph_state* s, double* corr, double* vol_re_im) {
  so3CombineCoef_fftw(s->bw, s->bw_out, s->bw - 1, s->sig_coef[0], s->sig_coef[1], s->pat_coef[0],
                      s->pat_coef[1], s->so3_coef);
  Inverse_SO3_Naive_fftw(s->bw_out, s->so3_coef, s->so3_sig, s->workspace1, s->workspace2_out,
                         s->workspace3_out, &s->inverse_so3, 1);
  const long nv = 8L * s->bw_out * s->bw_out * s->bw_out;
  for (long i = 0; i < nv; ++i) {
    const double re = s->so3_sig[i][0], im = s->so3_sig[i][1];
    if (corr) corr[i] = re * re + im * im;
    if (vol_re_im) {
      vol_re_im[2 * i] = re;
      vol_re_im[2 * i + 1] = im;
    }
  }
}

/* SOFT forward SHT of one real 2B x 2B signal. */
void ref_sht(int bw, const double* sig, double* re, double* im) {
  sph_state s;
  sph_init(&s, bw, bw);
  sph_transform_pair(&s, sig, sig);
  memcpy(re, s.sig_coef[0], sizeof(double) * bw * bw);
  memcpy(im, s.sig_coef[1], sizeof(double) * bw * bw);
  sph_free(&s);
}

/* C == 1: SphericalCorrelation::correlateSampledSignals on channel 0.
 * C >= 2: SphericalCorrelationLaplace::correlateSampledSignals.
 * f, g: C x 4B^2 doubles.  corr: (2 bw_out)^3; vol (optional): complex. */
void ref_spherical_correlation(int bw, int bw_out, int C, const double* f,
                               const double* g, double* corr, double* vol_re_im) {
  sph_state s;
  sph_init(&s, bw, bw_out);
  const size_t ns = (size_t)4 * bw * bw;
  const uint32_t nc = (uint32_t)(bw * bw);
  if (C == 1) {
    sph_transform_pair(&s, f, g);
  } else {
    double* fch = (double*)malloc(sizeof(double) * 2 * nc * C);
    double* gch = (double*)malloc(sizeof(double) * 2 * nc * C);
    double* tmp = (double*)malloc(sizeof(double) * 2 * nc);
    for (int c = 0; c < C; ++c) {
      sph_transform_pair(&s, f + ns * c, g + ns * c);
      /* shiftSignals: FFTShift of each real/imag array (std::rotate) */
      for (int side = 0; side < 2; ++side) {
        double* re = side == 0 ? s.sig_coef[0] : s.pat_coef[0];
        double* im = side == 0 ? s.sig_coef[1] : s.pat_coef[1];
        for (uint32_t i = 0; i < nc; ++i) {
          tmp[2 * i] = re[i];
          tmp[2 * i + 1] = im[i];
        }
        orc_fftshift(tmp, nc);
        memcpy((side == 0 ? fch : gch) + (size_t)2 * nc * c, tmp, sizeof(double) * 2 * nc);
      }
    }
    double* F = (double*)malloc(sizeof(double) * 2 * nc);
    double* G = (double*)malloc(sizeof(double) * 2 * nc);
    orc_fuse_channels_literal(fch, C, nc, 5, 4.0f, F);
    orc_fuse_channels_literal(gch, C, nc, 5, 4.0f, G);
    orc_ifftshift(F, nc);
    orc_ifftshift(G, nc);
    for (uint32_t i = 0; i < nc; ++i) {
      s.sig_coef[0][i] = F[2 * i];
      s.sig_coef[1][i] = F[2 * i + 1];
      s.pat_coef[0][i] = G[2 * i];
      s.pat_coef[1][i] = G[2 * i + 1];
    }
    free(F);
    free(G);
    free(fch);
    free(gch);
    free(tmp);
  }
  sph_correlate_inverse(&s, corr, vol_re_im);
  sph_free(&s);
}

/* ------------------------------------------------------------------------ */
/* Spatial correlation with the reference's buffer shapes.                  */
/* ------------------------------------------------------------------------ */
typedef struct {
  int N;
  long nv;
  fftw_complex *F, *G, *C;
  double *c, *f, *g;
  fftw_plan fp, gp, cp;
} spat_state;

static void spat_init(spat_state* s, int N) {
  s->N = N;
  s->nv = (long)N * N * N;
  s->F = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * s->nv);
  s->G = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * s->nv);
  s->C = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * s->nv);
  memset(s->F, 0, sizeof(fftw_complex) * s->nv);
  memset(s->G, 0, sizeof(fftw_complex) * s->nv);
  memset(s->C, 0, sizeof(fftw_complex) * s->nv);
  s->c = (double*)calloc(s->nv, sizeof(double));
  s->f = (double*)calloc(s->nv, sizeof(double));
  s->g = (double*)calloc(s->nv, sizeof(double));
  s->fp = fftw_plan_dft_r2c_3d(N, N, N, s->f, s->F, FFTW_ESTIMATE);
  s->gp = fftw_plan_dft_r2c_3d(N, N, N, s->g, s->G, FFTW_ESTIMATE);
  s->cp = fftw_plan_dft_c2r_3d(N, N, N, s->C, s->c, FFTW_ESTIMATE);
}

static void spat_free(spat_state* s) {
  fftw_free(s->F);
  fftw_free(s->G);
  fftw_free(s->C);
  fftw_destroy_plan(s->fp);
  fftw_destroy_plan(s->gp);
  fftw_destroy_plan(s->cp);
  free(s->c);
  free(s->f);
  free(s->g);
}

static void complex_mul_seq(const fftw_complex* F, const fftw_complex* G, fftw_complex* C, long n) {
  for (long i = 0; i < n; ++i) {
    C[i][0] = F[i][0] * G[i][0] - F[i][1] * (-G[i][1]);
    C[i][1] = F[i][0] * (-G[i][1]) + F[i][1] * G[i][0];
  }
}

/* laplace = 0: SpatialCorrelation on channel 0; 1: SpatialCorrelationLaplace. */
void ref_spatial_correlation(int N, int C, const double* f, const double* g,
                             int laplace, double* out) {
  spat_state s;
  spat_init(&s, N);
  const long nv = s.nv;
  if (!laplace) {
    memcpy(s.f, f, sizeof(double) * nv);
    memcpy(s.g, g, sizeof(double) * nv);
    fftw_execute(s.fp);
    fftw_execute(s.gp);
    complex_mul_seq(s.F, s.G, s.C, nv);
    fftw_execute(s.cp);
  } else {
    double* fch = (double*)malloc(sizeof(double) * 2 * nv * C);
    double* gch = (double*)malloc(sizeof(double) * 2 * nv * C);
    for (int c = 0; c < C; ++c) {
      memcpy(s.f, f + nv * c, sizeof(double) * nv);
      memcpy(s.g, g + nv * c, sizeof(double) * nv);
      fftw_execute(s.fp);
      fftw_execute(s.gp);
      orc_fftshift((double*)s.F, (size_t)nv);
      orc_fftshift((double*)s.G, (size_t)nv);
      memcpy(fch + 2 * nv * c, s.F, sizeof(fftw_complex) * nv);
      memcpy(gch + 2 * nv * c, s.G, sizeof(fftw_complex) * nv);
    }
    double* Ff = (double*)malloc(sizeof(double) * 2 * nv);
    double* Gf = (double*)malloc(sizeof(double) * 2 * nv);
    orc_fuse_channels_literal(fch, C, (uint32_t)nv, 5, 4.0f, Ff);
    orc_fuse_channels_literal(gch, C, (uint32_t)nv, 5, 4.0f, Gf);
    complex_mul_seq((fftw_complex*)Ff, (fftw_complex*)Gf, s.C, nv);
    orc_ifftshift((double*)s.C, (size_t)nv);
    fftw_execute(s.cp);
    free(fch);
    free(gch);
    free(Ff);
    free(Gf);
  }
  memcpy(out, s.c, sizeof(double) * nv);
  spat_free(&s);
}

/* ------------------------------------------------------------------------ */
/* kd-tree 1-NN (float L2, lowest index on ties) for the CPU baseline.      */
/* ------------------------------------------------------------------------ */
typedef struct {
  const float* p;
  int32_t* idx;
  int32_t* node_lo;
  int32_t* node_hi;
  int32_t* node_dim;
  float* node_split;
  int32_t* node_left;
  int32_t* node_right;
  int nn;
} kdtree;

static const float* g_sort_pts;
static int g_sort_dim;

static int cmp_idx(const void* a, const void* b) {
  const int32_t ia = *(const int32_t*)a, ib = *(const int32_t*)b;
  const float va = g_sort_pts[3 * ia + g_sort_dim], vb = g_sort_pts[3 * ib + g_sort_dim];
  if (va < vb) return -1;
  if (va > vb) return 1;
  return (ia > ib) - (ia < ib);
}

static int kd_build(kdtree* t, int lo, int hi) {
  const int id = t->nn++;
  t->node_lo[id] = lo;
  t->node_hi[id] = hi;
  t->node_left[id] = t->node_right[id] = -1;
  if (hi - lo <= 16) {
    t->node_dim[id] = -1;
    return id;
  }
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = lo; i < hi; ++i)
    for (int d = 0; d < 3; ++d) {
      const float v = t->p[3 * t->idx[i] + d];
      if (v < mn[d]) mn[d] = v;
      if (v > mx[d]) mx[d] = v;
    }
  int dim = 0;
  for (int d = 1; d < 3; ++d)
    if (mx[d] - mn[d] > mx[dim] - mn[dim]) dim = d;
  g_sort_pts = t->p;
  g_sort_dim = dim;
  qsort(t->idx + lo, (size_t)(hi - lo), sizeof(int32_t), cmp_idx);
  const int mid = (lo + hi) / 2;
  t->node_dim[id] = dim;
  t->node_split[id] = t->p[3 * t->idx[mid] + dim];
  const int l = kd_build(t, lo, mid);
  const int r = kd_build(t, mid, hi);
  t->node_left[id] = l;
  t->node_right[id] = r;
  return id;
}

static void kd_search(const kdtree* t, int node, const float* q, float* best, int32_t* bi) {
  if (t->node_dim[node] < 0) {
    for (int i = t->node_lo[node]; i < t->node_hi[node]; ++i) {
      const int32_t j = t->idx[i];
      const float dx = q[0] - t->p[3 * j], dy = q[1] - t->p[3 * j + 1], dz = q[2] - t->p[3 * j + 2];
      float r = 0.0f;
      r += dx * dx;
      r += dy * dy;
      r += dz * dz;
      if (r < *best || (r == *best && j < *bi)) {
        *best = r;
        *bi = j;
      }
    }
    return;
  }
  const int d = t->node_dim[node];
  const float diff = q[d] - t->node_split[node];
  const int first = diff < 0 ? t->node_left[node] : t->node_right[node];
  const int second = diff < 0 ? t->node_right[node] : t->node_left[node];
  kd_search(t, first, q, best, bi);
  if ((double)diff * diff <= (double)(*best) * (1.0 + 1e-5)) kd_search(t, second, q, best, bi);
}

static void ref_sample_cloud(const float* xyzi, size_t P, const float* refl, int bw,
                             float max_sq, double* out) {
  const size_t nq = (size_t)4 * bw * bw;
  float* grid = (float*)malloc(sizeof(float) * 3 * nq);
  orc_dh_grid(bw, grid);
  float* proj = (float*)malloc(sizeof(float) * 3 * (P ? P : 1));
  double* rng = (double*)malloc(sizeof(double) * (P ? P : 1));
  orc_project(xyzi, 4, P, proj, rng);
  kdtree t;
  memset(&t, 0, sizeof(t));
  t.p = proj;
  t.idx = (int32_t*)malloc(sizeof(int32_t) * (P ? P : 1));
  for (size_t i = 0; i < P; ++i) t.idx[i] = (int32_t)i;
  const size_t maxn = 2 * (P / 8 + 2) + 16;
  t.node_lo = (int32_t*)malloc(sizeof(int32_t) * maxn);
  t.node_hi = (int32_t*)malloc(sizeof(int32_t) * maxn);
  t.node_dim = (int32_t*)malloc(sizeof(int32_t) * maxn);
  t.node_split = (float*)malloc(sizeof(float) * maxn);
  t.node_left = (int32_t*)malloc(sizeof(int32_t) * maxn);
  t.node_right = (int32_t*)malloc(sizeof(int32_t) * maxn);
  if (P > 0) kd_build(&t, 0, (int)P);
  for (size_t i = 0; i < nq; ++i) {
    float best = INFINITY;
    int32_t bi = -1;
    if (P > 0) kd_search(&t, 0, grid + 3 * i, &best, &bi);
    double r = 0, it = 0, rf = 0;
    if (bi >= 0 && !(best > max_sq)) {
      r = rng[bi];
      it = xyzi[4 * (size_t)bi + 3];
      rf = refl ? refl[bi] : 0.0;
    }
    out[i] = r;
    out[nq + i] = it;
    out[2 * nq + i] = rf;
    out[3 * nq + i] = 0.0;
  }
  free(grid);
  free(proj);
  free(rng);
  free(t.idx);
  free(t.node_lo);
  free(t.node_hi);
  free(t.node_dim);
  free(t.node_split);
  free(t.node_left);
  free(t.node_right);
}

int ref_register_pair_mode(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                           const float* src_xyzi, size_t Ps, const float* src_refl,
                           int bw, int N, int lo, int hi, float max_sq, int threads, int sph_mode,
                           uint32_t* rot_bin, uint32_t* voxel, double* pose6);

/* Whole registration on the CPU: returns rotation bin and translation voxel;
 * pose6 = {x, y, z rotation angles (XYZ), tx, ty, tz}. */
int ref_register_pair(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                      const float* src_xyzi, size_t Ps, const float* src_refl,
                      int bw, int N, int lo, int hi, float max_sq, int threads,
                      uint32_t* rot_bin, uint32_t* voxel, double* pose6) {
  return ref_register_pair_mode(tgt_xyzi, Pt, tgt_refl, src_xyzi, Ps, src_refl, bw, N, lo, hi, max_sq, threads,
                                0, rot_bin, voxel, pose6);
}

/* sph_mode 0: SphOptRegistration (sph-opt-registration.cc:34-132: four
 * channels, SphericalCorrelationLaplace); 1: SphRegistration
 * (sph-registration.cc:82-198: SphericalCorrelation::correlateSignals on the
 * 0.6 intensity + 0.4 range signal of each direction). */
int ref_register_pair_mode(const float* tgt_xyzi, size_t Pt, const float* tgt_refl,
                           const float* src_xyzi, size_t Ps, const float* src_refl,
                           int bw, int N, int lo, int hi, float max_sq, int threads, int sph_mode,
                           uint32_t* rot_bin, uint32_t* voxel, double* pose6) {
  fftw_plan_with_nthreads(threads);
  const size_t ns = (size_t)4 * bw * bw;
  double* f = (double*)malloc(sizeof(double) * 4 * ns);
  double* h = (double*)malloc(sizeof(double) * 4 * ns);
  ref_sample_cloud(tgt_xyzi, Pt, tgt_refl, bw, max_sq, f);
  ref_sample_cloud(src_xyzi, Ps, src_refl, bw, max_sq, h);
  const long nvol = 8L * bw * bw * bw;
  double* corr = (double*)malloc(sizeof(double) * nvol);
  if (sph_mode == 1) {
    for (size_t i = 0; i < ns; ++i) {
      f[i] = 0.6 * f[ns + i] + 0.4 * f[i];
      h[i] = 0.6 * h[ns + i] + 0.4 * h[i];
    }
    ref_spherical_correlation(bw, bw, 1, f, h, corr, NULL);
  } else {
    ref_spherical_correlation(bw, bw, 4, f, h, corr, NULL);
  }
  const uint64_t bin = orc_argmax(corr, (uint64_t)nvol);
  double zyz[3], q[4], xyz[3];
  orc_bin_to_zyz((uint32_t)bin, (uint32_t)bw, zyz);
  orc_zyz_to_quat(zyz, q);
  orc_quat_to_xyz(q, xyz);
  float T[12];
  orc_rotation_xyz((float)xyz[0], (float)xyz[1], (float)xyz[2], T);
  float* rot = (float*)malloc(sizeof(float) * 4 * (Ps ? Ps : 1));
  memcpy(rot, src_xyzi, sizeof(float) * 4 * Ps);
  orc_transform(rot, Ps, T);
  const long nv = (long)N * N * N;
  double* fv = (double*)malloc(sizeof(double) * 4 * nv);
  double* gv = (double*)malloc(sizeof(double) * 4 * nv);
  orc_discretize(tgt_xyzi, Pt, tgt_refl, NULL, N, lo, hi, fv);
  orc_discretize(rot, Ps, src_refl, NULL, N, lo, hi, gv);
  double* c = (double*)malloc(sizeof(double) * nv);
  ref_spatial_correlation(N, 4, fv, gv, 1, c);
  const uint64_t vox = orc_argmax(c, (uint64_t)nv);
  uint32_t ijk[3];
  orc_ind2sub((uint32_t)vox, (uint32_t)N, (uint32_t)N, ijk);
  *rot_bin = (uint32_t)bin;
  *voxel = (uint32_t)vox;
  pose6[0] = xyz[0];
  pose6[1] = xyz[1];
  pose6[2] = xyz[2];
  for (int a = 0; a < 3; ++a) pose6[3 + a] = orc_translation_from_index((double)ijk[a], (uint32_t)N, lo, hi);
  free(f);
  free(h);
  free(corr);
  free(rot);
  free(fv);
  free(gv);
  free(c);
  return 0;
}
