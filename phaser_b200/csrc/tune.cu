// Autotuner of the per-shape launch parameters (phgpu_tuning_*,
// phgpu_autotune).
//
// Parameters: the ky tile width of the translation z pass (k_fuse_z), the beta
// tile of the SO(3) alpha transform (k_so3_fft_a), the degree chunk of the
// tensor-core synthesis (k_so3_synth_tc) and the radix order of runtime FFT
// plans (lengths without a compile-time plan).  The search is coordinate-wise:
// each parameter's candidates are timed in turn, the others held at their
// current values, on registrations of a caller-supplied pair with the
// context's own buffers, by the per-stage CUDA events the context records on
// each stage's stream (phgpu_profile_*).
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>
#include <vector>

#include "../../include/phaser_gpu.h"
#include "ctx.h"

using namespace phgpu;

namespace {

bool compile_time_length(int n) {
  return n == 64 || n == 128 || n == 200 || n == 256 || n == 320 || n == 512;
}

// Whether any of the context's transforms runs on a runtime plan.
bool has_runtime_plan(const phgpu_ctx* c) {
  if (!compile_time_length(2 * c->bw) || !compile_time_length(2 * c->bw_out) || !compile_time_length(c->N))
    return true;
  if (c->has_sp_half && !compile_time_length(c->N / 2)) return true;
  return c->pad && (!compile_time_length(c->M) || (c->has_pad_half && !compile_time_length(c->M / 2)));
}

void apply_radix_order(phgpu_ctx* c, int order) {
  for (FftPlan* p : {&c->plan_s2, &c->plan_so3, &c->plan_sp, &c->plan_sp_half, &c->plan_pad, &c->plan_pad_half}) {
    if (p->n < 1) continue;
    FftPlan q = *p;
    if (fft_plan_radices(p->n, order, &q)) *p = q;
  }
}

int tuning_valid(const phgpu_ctx* c, const phgpu_tuning& t) {
  const uint32_t f = t.fuse_z_tile;
  if (f && !(f == 2 || f == 4 || f == 8 || f == 16)) return 0;
  if (t.so3_beta_tile && !so3_beta_tile_ok(c->bw_out, (int)t.so3_beta_tile)) return 0;
  if (t.tc_chunk) {
    if (t.tc_chunk != 16 && t.tc_chunk != 32) return 0;
    if (c->prm.precision != PHGPU_PRECISION_FP32 &&
        !so3_tc_supported(c->bw_out, 1, (int)c->prm.precision, (int)t.tc_chunk))
      return 0;
  }
  return t.radix_order <= 2;
}

}  // namespace

int phgpu_tuning_get(const phgpu_ctx* ctx, phgpu_tuning* out) {
  if (!ctx || !out) return PHGPU_ERR_INVALID;
  *out = ctx->tune;
  return PHGPU_OK;
}

int phgpu_tuning_set(phgpu_ctx* ctx, const phgpu_tuning* t) {
  if (!ctx || !t) return PHGPU_ERR_INVALID;
  if (!tuning_valid(ctx, *t)) {
    ctx->err = "tuning value out of range for this shape";
    return PHGPU_ERR_INVALID;
  }
  if (t->radix_order != ctx->tune.radix_order) apply_radix_order(ctx, (int)t->radix_order);
  ctx->tune = *t;
  return PHGPU_OK;
}

int phgpu_autotune(phgpu_ctx* ctx, const phgpu_cloud* target, const phgpu_cloud* source, uint32_t reps,
                   phgpu_tuning* best, double* ms_per_pair) {
  if (!ctx || !target || !source || reps < 1) return PHGPU_ERR_INVALID;
  const bool prof_was = ctx->prof_on;
  phgpu_profile_enable(ctx, 1);
  const int n_st = phgpu_profile_stage_count();
  std::vector<double> ms(n_st);
  std::vector<unsigned long long> calls(n_st);
  phgpu_pose pose;
  // device time of `stage` per registration (all stages when stage < 0)
  auto measure = [&](int stage, double* out) -> int {
    int rc = phgpu_register_pair(ctx, target, source, &pose);  // warm-up
    if (rc == PHGPU_OK) rc = phgpu_profile_read(ctx, ms.data(), calls.data(), n_st);
    for (uint32_t r = 0; r < reps && rc == PHGPU_OK; ++r) rc = phgpu_register_pair(ctx, target, source, &pose);
    if (rc == PHGPU_OK) rc = phgpu_profile_read(ctx, ms.data(), calls.data(), n_st);
    if (rc != PHGPU_OK) return rc;
    double t = 0.0;
    for (int s = 0; s < n_st; ++s)
      if (stage < 0 ? s != PS_UPLOAD : s == stage) t += ms[s];
    *out = t / reps;
    return PHGPU_OK;
  };
  struct Param {
    uint32_t phgpu_tuning::*field;
    std::vector<uint32_t> cand;
    int stage;
  };
  std::vector<Param> params = {{&phgpu_tuning::fuse_z_tile, {0, 2, 4, 8, 16}, PS_FUSE_Z},
                               {&phgpu_tuning::so3_beta_tile, {8, 16, 32}, PS_SO3_FFT}};
  if (ctx->prm.precision != PHGPU_PRECISION_FP32) params.push_back({&phgpu_tuning::tc_chunk, {16, 32}, PS_SO3_SYNTH});
  if (has_runtime_plan(ctx)) params.push_back({&phgpu_tuning::radix_order, {0, 1, 2}, -1});
  phgpu_tuning cur = ctx->tune;
  int rc = PHGPU_OK;
  for (const Param& p : params) {
    uint32_t best_v = cur.*(p.field);
    double best_t = DBL_MAX;
    for (uint32_t v : p.cand) {
      phgpu_tuning t = cur;
      t.*(p.field) = v;
      if (!tuning_valid(ctx, t)) continue;
      phgpu_tuning_set(ctx, &t);
      double tm = 0.0;
      rc = measure(p.stage, &tm);
      if (rc != PHGPU_OK) break;
      if (tm < best_t) {
        best_t = tm;
        best_v = v;
      }
    }
    if (rc != PHGPU_OK) break;
    cur.*(p.field) = best_v;
    phgpu_tuning_set(ctx, &cur);
  }
  double total = 0.0;
  if (rc == PHGPU_OK) rc = measure(-1, &total);
  phgpu_profile_enable(ctx, prof_was ? 1 : 0);
  if (rc != PHGPU_OK) return rc;
  if (best) *best = cur;
  if (ms_per_pair) *ms_per_pair = total;
  return PHGPU_OK;
}
