// Test-only library (built by tests/test_gpu_fft_engines.py, linked against
// the product library for the FFT plans): self-test of the shared-memory FFT
// engines, phgpu_selftest_fft(n, ntrans, inverse, columns, engine, data),
// which transforms ntrans sequences of length n (complex interleaved, natural
// order, sequence-major, in place in `data`); engine 0 = runtime plan,
// 1 = compile-time plan, 2 = register-tail plan.  Forward = exp(-2 pi i jk/n),
// inverse = exp(+2 pi i jk/n), both unnormalised.  One block
// transforms `ntrans` sequences of length n held in shared memory as rows
// (stride n + 1) or columns (stride ntrans), through the runtime plan, the
// compile-time plan or the register-tail plan.  Input and output are in
// natural order; digit-reversed spectra are mapped with the plan.
#include <cuda_runtime.h>

#include <string>

#include "phaser_gpu.h"
#include "fft2.cuh"
#include "kernels.h"

namespace phgpu {
bool make_fft_plan(int n, FftPlan* p, float2** d_tw, std::string* err);
}

namespace phgpu {

template <int NF, int ENGINE, bool INV, bool COL>
__global__ void __launch_bounds__(1024) k_selftest_fft(int n, int ntrans, const float2* __restrict__ in, float2* __restrict__ out, FftPlan p) {
  extern __shared__ float2 buf[];
  const int stride = COL ? ntrans : n + 1;
  auto at = [&](int t, int i) -> float2& { return COL ? buf[t + i * stride] : buf[t * stride + i]; };
  for (int e = threadIdx.x; e < ntrans * n; e += blockDim.x) {
    const int t = e / n, i = e % n;
    // inverse transforms read digit-reversed input
    const int pos = INV ? freq2pos<NF>(i, p) : i;
    at(t, pos) = in[e];
  }
  __syncthreads();
  if constexpr (ENGINE == 2) {
    fft_tail<NF, INV, COL>(buf, ntrans, stride, p.tw);
  } else if constexpr (ENGINE == 1) {
    if (COL)
      fft_fixed<NF, INV, -2>(buf, ntrans, 1, stride, p.tw);
    else
      fft_fixed<NF, INV, -1>(buf, ntrans, stride, 1, p.tw);
  } else {
    if (COL)
      fft_smem<INV>(buf, ntrans, 1, stride, p);
    else
      fft_smem<INV>(buf, ntrans, stride, 1, p);
  }
  for (int e = threadIdx.x; e < ntrans * n; e += blockDim.x) {
    const int t = e / n, i = e % n;
    const int pos = INV ? i : freq2pos<NF>(i, p);
    out[e] = at(t, pos);
  }
}

template <int NF, int ENGINE>
static cudaError_t run_selftest(int n, int ntrans, int inverse, int columns, const float2* din, float2* dout,
                                const FftPlan& p) {
  const int threads = ENGINE == 2 ? tail_threads<NF>() : 512;
  const size_t sm = (size_t)ntrans * (n + 1) * sizeof(float2);
  if (inverse) {
    if (columns) {
      cudaFuncSetAttribute(k_selftest_fft<NF, ENGINE, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      k_selftest_fft<NF, ENGINE, true, true><<<1, threads, sm>>>(n, ntrans, din, dout, p);
    } else {
      cudaFuncSetAttribute(k_selftest_fft<NF, ENGINE, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      k_selftest_fft<NF, ENGINE, true, false><<<1, threads, sm>>>(n, ntrans, din, dout, p);
    }
  } else {
    if (columns) {
      cudaFuncSetAttribute(k_selftest_fft<NF, ENGINE, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      k_selftest_fft<NF, ENGINE, false, true><<<1, threads, sm>>>(n, ntrans, din, dout, p);
    } else {
      cudaFuncSetAttribute(k_selftest_fft<NF, ENGINE, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      k_selftest_fft<NF, ENGINE, false, false><<<1, threads, sm>>>(n, ntrans, din, dout, p);
    }
  }
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace phgpu

using namespace phgpu;

extern "C" int phgpu_selftest_fft(int n, int ntrans, int inverse, int columns, int engine, float* data) {
  if (n < 1 || ntrans < 1 || !data || (size_t)ntrans * (n + 1) * sizeof(float2) > 227 * 1024) return PHGPU_ERR_INVALID;
  FftPlan p;
  float2* tw = nullptr;
  std::string err;
  if (!make_fft_plan(n, &p, &tw, &err)) return PHGPU_ERR_INVALID;
  const size_t bytes = sizeof(float2) * (size_t)n * ntrans;
  float2 *din = nullptr, *dout = nullptr;
  if (cudaMalloc(&din, bytes) != cudaSuccess || cudaMalloc(&dout, bytes) != cudaSuccess) {
    cudaFree(din);
    cudaFree(tw);
    return PHGPU_ERR_MEMORY;
  }
  cudaMemcpy(din, data, bytes, cudaMemcpyHostToDevice);
  cudaError_t e = cudaErrorInvalidValue;
  int rc = PHGPU_OK;
  if (engine == 0) {
    e = run_selftest<0, 0>(n, ntrans, inverse, columns, din, dout, p);
  } else {
    switch (n) {
#define PHGPU_SELFTEST_CASE(NN)                                                   \
  case NN:                                                                        \
    e = engine == 2 ? run_selftest<NN, 2>(n, ntrans, inverse, columns, din, dout, p) \
                    : run_selftest<NN, 1>(n, ntrans, inverse, columns, din, dout, p); \
    break;
      PHGPU_SELFTEST_CASE(32)
      PHGPU_SELFTEST_CASE(64)
      PHGPU_SELFTEST_CASE(100)
      PHGPU_SELFTEST_CASE(128)
      PHGPU_SELFTEST_CASE(200)
      PHGPU_SELFTEST_CASE(256)
      PHGPU_SELFTEST_CASE(512)
#undef PHGPU_SELFTEST_CASE
      case 320:  // compile-time plan only (no register-tail plan)
        if (engine == 1)
          e = run_selftest<320, 1>(n, ntrans, inverse, columns, din, dout, p);
        else
          rc = PHGPU_ERR_INVALID;
        break;
      default:
        rc = PHGPU_ERR_INVALID;
    }
  }
  if (rc == PHGPU_OK) {
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
      rc = PHGPU_ERR_CUDA;
    else
      cudaMemcpy(data, dout, bytes, cudaMemcpyDeviceToHost);
  }
  cudaFree(din);
  cudaFree(dout);
  cudaFree(tw);
  return rc;
}
