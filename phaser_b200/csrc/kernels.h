// Internal launch interface of the PHASER registration kernels.  Host code in
// capi.cu owns every buffer; kernels only see raw device pointers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace phgpu {

// Number of kernels this library has launched (all contexts).
extern std::atomic<unsigned long long> g_launch_count;
// > 0 while this thread captures a CUDA graph (its kernels are counted when
// the graph is launched)
extern thread_local int g_capture_depth;
inline void count_launches(int n) {
  if (!g_capture_depth) g_launch_count.fetch_add((unsigned long long)n, std::memory_order_relaxed);
}

// ------------------------------------------------------------ S^2 sampling
struct SampleArgs {
  const float4* xyzi;   // [n_points] x, y, z, intensity
  const float* refl;    // [n_points] or null
  const float* amb;     // [n_points] or null
  int n_points;
  int max_points;       // scratch sizing
  const float4* grid;   // [n_queries] DH grid directions (host-computed)
  int n_queries;
  int n2b = 0;          // 2B: grid is the 2B x 2B DH grid (n_queries = n2b^2)
  float max_sq;         // squared voxel size (rejection threshold)
  int n_out_ch;         // channels written (1..4)
  float* out;           // [n_out_ch][n_queries]
  int32_t* nn_idx;      // [n_queries] or null
  void* scratch;        // sampler_scratch_bytes(max_points, >= n_queries)
  const uint32_t* n_dev = nullptr;  // when set: the point count is read from device memory (n_points = capacity)
};
size_t sampler_scratch_bytes(int max_points, int max_queries);
cudaError_t launch_sample(const SampleArgs& a, cudaStream_t st);

// ------------------------------------------------------------ forward SHT
// Legendre table: for m in [0,B), l in [m,B), k in [0,2B):
//   T[off(m) + (l-m)*2B + k] = w_k * Pbar_l^m(cos theta_k)
size_t legendre_table_entries(int bw);
cudaError_t launch_legendre_table(int bw, const double* weights_dev, float* table, cudaStream_t st);

// Both sides at once: signal (side, c) at signal + side * side_stride + c (2B)^2.
constexpr int kMaxWaveSht = 32;  // requests per batched Legendre launch (kMaxWave)
struct ShtArgs {
  int bw;
  int n_data;             // channels per side (1..4)
  size_t side_stride;     // floats between the two sides' grids
  const float* signal;    // [side][c][2B][2B]
  const FftPlan* plan;    // length 2B
  const float* table;     // Legendre table
  float2* fphi;           // scratch [side][c][B (m)][2B (k)], sht_scratch_entries(B) complex
  float2* coef;           // [side][c][B (l)][B (m>=0)]
  const float* table_tc = nullptr;  // tensor-core layout of the table (legendre_tc_floats): the
                                    // contraction runs on the tensor cores when set
  int precision = 0;                // kSo3Tf32x3 / kSo3Bf16x3 with table_tc
  int tc_chunk = 0;
  unsigned long long* status = nullptr;
};
// The Legendre contraction of several requests (one launch): fphi / coef per request.
struct ShtBatch {
  int count;
  const float2* fphi[kMaxWaveSht];
  float2* coef[kMaxWaveSht];
};
size_t sht_scratch_entries(int bw);
cudaError_t launch_sht(const ShtArgs& a, cudaStream_t st);      // phi pass + Legendre contraction
cudaError_t launch_sht_phi(const ShtArgs& a, cudaStream_t st);  // phi pass alone
cudaError_t sht_init_attributes();  // once per device
// Tensor-core Legendre contraction (k_sht.cu): the table relaid [m][k / 4][l][4].
size_t legendre_tc_floats(int bw);
cudaError_t launch_legendre_tc_layout(int bw, const float* table, float* table_tc, cudaStream_t st);
bool sht_leg_tc_supported(int bw, int count, int precision);
cudaError_t launch_sht_leg_tc(int bw, int n_data, const ShtBatch& b, const float* table_tc, int precision, int chunk,
                              unsigned long long* status, cudaStream_t st);

struct FuseS2Args {
  int bw;
  int n_data_ch;          // channels with data per side
  int n_total_ch;         // divisor of the channel mean (reference channel count)
  int laplace;            // 0: take channel 0 (plain SphericalCorrelation)
  int lowpass;            // 1: channel 0, coefficients at shifted positions outside [lp_lo, lp_hi) zeroed
  uint32_t lp_lo, lp_hi;
  FusionBands bands;      // for n = B^2
  const float2* coef;     // [2][n_data_ch][B][B]   (side-major)
  float2* fused;          // [2][B (l)][2B-1 (m + B - 1)]
  int count = 0;          // > 0: requests of one launch, coef_b / fused_b per request (else coef / fused)
  const float2* coef_b[32];
  float2* fused_b[32];
};
cudaError_t launch_fuse_s2(const FuseS2Args& a, cudaStream_t st);
// out[side][k] = 0.6 * intensity + 0.4 * range of samples [side][c][n] (n = 4B^2)
cudaError_t launch_mix_signal(const float* samples, size_t side_stride, int n, float* out, cudaStream_t st);

// ------------------------------------------------------------ SO(3)
// Requests of one shape processed by one launch (a wave of the server).
constexpr int kMaxWave = 32;
struct So3Out {
  float2* S;                   // [2 bw_out (a)][bw_out (b)][2 bw_out (beta)]
  unsigned long long* argmax;  // packed (value^2, index)
  float* volume;               // optional (2 bw_out)^3 |z|^2, [beta][alpha][gamma]
};
struct So3Batch {
  int count;                      // requests (1..kMaxWave)
  const float2* fused[kMaxWave];  // [2][bw_in][2 bw_in - 1] per request
  So3Out out[kMaxWave];
};
struct So3Args {
  int bw_in;              // degree limit
  int bw_out;             // output grid 2*bw_out
  const double* beta_tab; // [3][2 bw_out]: cos(beta_k), log cos(beta_k / 2), log sin(beta_k / 2)
  const double* wig_tab;  // so3_wigner_table(bw_in): recurrence square roots, per-degree factors
  const FftPlan* plan;    // length 2 bw_out
  So3Batch batch;
  int beta_tile = 0;      // betas per alpha-FFT block (8, 16, 32; 0 = 16): tuned
  int tc_chunk = 0;       // degrees per tensor-core chunk (16, 32; 0 = the largest that fits): tuned
};
bool so3_beta_tile_ok(int bw_out, int wt);
cudaError_t launch_so3_synth(const So3Args& a, cudaStream_t st);  // coefficient product + FP32 Wigner synthesis
cudaError_t launch_so3_fft(const So3Args& a, cudaStream_t st);    // alpha FFT + gamma C2R + argmax
cudaError_t so3_init_attributes();  // once per device
void so3_beta_table(int bw_out, double* host_tab);  // fills the [3][2 bw_out] beta_tab on the host
void so3_wigner_table(int bw_in, std::vector<double>& host_tab);  // recurrence tables of the synthesis

// Tensor-core synthesis (k_so3_tc.cu) from a Wigner-d table generated once in
// FP64 and stored as FP32: per order class (p, q) a [nl_pad / 4][2 bw_out][4]
// block (nl_pad = bw_in - q rounded up to 8), i.e. 16-byte groups of four
// degrees for every beta, the operand layout of the matrix instructions.
enum So3Precision { kSo3Fp32 = 0, kSo3Tf32x3 = 1, kSo3Bf16x3 = 2 };
struct So3Table {
  const float* table;       // Wigner-d values of every class
  const size_t* class_off;  // [classes] float offset of each class's block
  int precision;            // kSo3Tf32x3 or kSo3Bf16x3
};
// Offsets of every class's block (host) and the table's float count.
size_t so3_table_layout(int bw_in, int bw_out, std::vector<size_t>* class_off);
cudaError_t launch_so3_table(int bw_in, int bw_out, const double* beta_tab, const double* wig_tab,
                             const size_t* class_off, float* table, cudaStream_t st);
// Whether a launch of `count` requests fits the tensor-core kernel's shared
// and tensor memory (bw_out <= 256, count <= kMaxWave).
bool so3_tc_supported(int bw_out, int count, int precision, int chunk = 0);
cudaError_t launch_so3_synth_tc(const So3Args& a, const So3Table& t, unsigned long long* status, cudaStream_t st);
cudaError_t so3_tc_init_attributes();

// Rotation pose of each request's SO(3) argmax on the device (k_pose.cu):
// T[r] receives the float 3x4 transform RotateAroundXYZ applies to the source.
struct PoseBatch {
  int count;
  uint32_t bw_out;
  const unsigned long long* argmax[kMaxWave];
  float* T[kMaxWave];  // 12 floats each
};
cudaError_t launch_pose(const PoseBatch& b, cudaStream_t st);

// ------------------------------------------------------------ spatial
struct VoxelArgs {
  const float4* xyzi;
  const float* refl;
  const float* amb;
  int n_points;
  int N;
  const float* edges;     // [N]
  int has_T;
  float T[12];            // 3x4 row-major, applied in PCL order
  int n_data_ch;          // channels accumulated (1..4) in order {int, range, refl, amb}
  float* grids;           // [n_data_ch + 1][N^3] sums, last = count
  uint32_t* lin_out;      // optional per-point linear index (or 0xffffffff)
  uint8_t* rowlive;       // optional [N (z)][N (x)]: set to 1 for every row a point lands in
  const float* T_dev = nullptr;     // when set: the 3x4 transform is read from device memory (has_T ignored)
  const uint32_t* n_dev = nullptr;  // when set: the point count is read from device memory (n_points = capacity)
};
cudaError_t launch_voxelize(const VoxelArgs& a, cudaStream_t st);
// Zeroes what one voxelisation wrote: planes [0, n_planes) at every point's
// voxel (lin[i] != 0xffffffff) and the point's row flag.
cudaError_t launch_clear_voxels(const uint32_t* lin, int n_points, float* grids, size_t nv, int n_planes,
                                uint8_t* rowlive, int N, cudaStream_t st, const uint32_t* n_dev = nullptr);

struct SpatialArgs {
  int N;
  int n_data_ch;          // channels per side with data
  int n_total_ch;         // mean divisor
  int laplace;            // 0: plain SpatialCorrelation on channel 0
  int lowpass;            // 1 (with laplace 0): channel 1, products outside the shifted cube zeroed
  uint32_t lp_lo, lp_hi;  // cube [lp_lo, lp_hi]^3 of subscripts
  FusionBands bands;      // for n = N^3
  const float* grids_f;   // [n_data_ch + 1][N^3] target sums + count (normalised here)
  const float* grids_g;   // source
  int grids_are_means;    // 1: grids already hold values (no count plane)
  const uint8_t* rowlive_f;  // optional row flags of the grids (rows never flagged are all zero)
  const uint8_t* rowlive_g;
  uint8_t* slab_nz;       // optional [2 n_data_ch][N] per spectrum array: 0 where the z-slab is known
                          // to hold zeros (the z-slab forward then skips a slab that stays zero,
                          // and keeps the flags); null: every slab is written
  float2* spec;           // [2 n_data_ch][N (z)][N (x)][H2p (ky)]
  float2* cspec;          // [N][N][H2p]
  const FftPlan* plan;    // length N
  const FftPlan* plan_half;  // length N/2 (z-slab kernels), may be null
  unsigned long long* argmax;
  float* volume;          // optional N^3 correlation, [z][x][y]
  unsigned long long* status;  // bit 0: a bulk-copy wait gave up (result invalid)
  uint32_t argmax_limit = 0;   // argmax over indices < limit (0: all)
  int fuse_tile = 0;           // ky columns per k_fuse_z block (2, 4, 8, 16; 0 = widest with two blocks per SM): tuned
};
// Whether a k_fuse_z tile of wt ky columns fits shared memory for N and A arrays.
bool fuse_z_tile_ok(int N, int A, int wt);
cudaError_t launch_spatial_forward(const SpatialArgs& a, int side, cudaStream_t st);
cudaError_t launch_spatial_combine(const SpatialArgs& a, cudaStream_t st);
cudaError_t launch_spatial_fuse_z(const SpatialArgs& a, cudaStream_t st);   // z FFTs + fusion + cross power
cudaError_t launch_spatial_inverse(const SpatialArgs& a, cudaStream_t st);  // inverse x + C2R y + argmax
cudaError_t spatial_init_attributes();  // once per device
// ------------------------------------------------------------ zero-padded translation
// The reference's padded spatial correlation (spatial-correlation.cc:11-45,
// 142-161,223-230): the product of the (fused) N-sized spectra is scattered
// to computeZeroPaddedIndex positions of an M = N + 2 pad cube and inverted
// at M.  See k_spatial_pad.cu.
struct PadArgs {
  int N, M, pad;
  int mode;               // 0 plain (channel 0), 1 Laplace fusion, 2 low-pass (channel 1, index cube)
  int n_ch;               // channels fused per side (mode 1: all channels, zero ones included)
  int n_spec;             // channels with spectra in spec (mode 1; the others are zero)
  int spec_ch;            // channels per side in the spec layout
  int first_ch;           // spec channel read by modes 0 and 2
  const float2* spec;     // [2][spec_ch][N (z pos)][N (x pos)][H2p]: full 3-D spectra
  const float2* prev_f;   // last channel of the previous call (mode 1), null = zero
  const float2* prev_g;
  int x_natural_N;        // spec x positions: 1 natural, 0 digit-reversed
  int x_natural_M;        // cspec_pad x positions expected by the inverse at M
  FftPlan planN, planM;   // z positions (both digit-reversed)
  FusionBands bands;      // n = N^3
  uint32_t lp_lo, lp_hi;  // mode 2 index cube
  float inv_total;        // 1 / channel count (MEAN)
  float2* cspec;          // [M (z pos)][M (x pos)][H2p(M)], zeroed by the caller
};
// Forward (INV = 0) or inverse z transform of n_arrays [n][nx][H2p] arrays
// (z natural <-> z digit-reversed), columns ky < H.
cudaError_t launch_pad_zfft(float2* base, size_t array_stride, int n_arrays, int n, int nx, int H, int inverse,
                            const FftPlan& plan, cudaStream_t st);
cudaError_t launch_pad_fuse(const PadArgs& a, cudaStream_t st);

// Row length of the half spectra: N/2 + 1 rounded up to 8 complex (64 B).
__host__ __device__ inline int spatial_h2p(int N) { return ((N / 2 + 1) + 7) / 8 * 8; }
// True when the fused z-slab kernels handle this N (the slab fits in shared memory).
bool spatial_slab_path(int N);

}  // namespace phgpu
