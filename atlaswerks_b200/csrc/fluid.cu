// fluid.cu — fused FFT kernels of the fluid operator solve (see fluid.cuh).
//
// Reference behaviour (Algorithms/Common/DiffOper.cxx:825-905 on the CPU,
// CUDACommon/src/cudaFFTSolver.cu:675-704 on the old GPU path): the force is
// scaled by 1/N, transformed, multiplied per wavenumber by L(k)^-1 (or L(k)),
// and transformed back, with
//   lambda = -alpha*(cx+cy+cz) + gamma,  L_ii = lambda - beta*c_i,
//   L_ij = beta*s_i*s_j,  c = (2cos(2 pi k/n) - 2)/sp^2,  s = sin(2 pi k/n)/sp
// (LUT: DiffOper.cxx:590-639; Cholesky: DiffOper.cxx:1005-1083). Here the
// 1/N scaling is folded into the per-wavenumber step.
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "bulk.cuh"
#include "fluid.cuh"
#include "tma_host.cuh"
#include "fluid_fast.cuh"

namespace aw {

namespace {

// Radix plan: as many 8s as possible, a 4 instead of an 8*2 tail, then 3,
// then any remaining prime (direct DFT).
bool factorize(int n, FFTAxis &ax) {
  int e = 0, m = n;
  while (m % 2 == 0) { m /= 2; ++e; }
  std::vector<int> r;
  int e8 = e / 3, rem = e % 3;
  if (rem == 1 && e8 > 0) { --e8; r.push_back(4); r.push_back(4); rem = 0; }
  for (int i = 0; i < e8; ++i) r.insert(r.begin(), 8);
  if (rem == 2) r.push_back(4);
  if (rem == 1) r.push_back(2);
  while (m % 3 == 0) { r.push_back(3); m /= 3; }
  for (int p = 5; m > 1; p += 2)
    while (m % p == 0) { r.push_back(p); m /= p; }
  if ((int)r.size() > kMaxStages) return false;
  ax.n = n;
  ax.nstages = (int)r.size();
  for (int i = 0; i < ax.nstages; ++i) ax.radix[i] = r[i];
  return true;
}

void fill_twiddles(int n, std::vector<float2> &out) {
  for (int m = 0; m < n; ++m) {
    const double a = -2.0 * M_PI * (double)m / (double)n;
    out.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
  }
}

// reference LUT, computed in double and stored as float like DiffOperT<float>
void fill_lut(int n, double sp, std::vector<float> &out) {
  const double s = 2.0 * M_PI / n;
  for (int k = 0; k < n; ++k) out.push_back((float)((2.0 * std::cos(s * k) - 2.0) / (sp * sp)));
  for (int k = 0; k < n; ++k) out.push_back((float)(std::sin(s * k) / sp));
}

template <class Src>
__global__ void __launch_bounds__(256) k_fft_xy_fwd(FluidPlan p, Src src) {
  extern __shared__ float2 sm[];
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nxh = p.nxh;
  const int P = p.pairs_per_batch, Q = p.cols_per_batch;
  const int ws = max(P * nx, Q * ny);
  float2 *C = sm;
  float2 *A = C + ny * nxh;
  float2 *B = A + ws;
  const int npairs = (ny + 1) >> 1;
  for (int p0 = 0; p0 < npairs; p0 += P) {
    const int pb = min(P, npairs - p0);
    for (int t = threadIdx.x; t < pb * nx; t += blockDim.x) {
      const int b = t / nx, x = t - b * nx;
      const int y0 = 2 * (p0 + b), y1 = y0 + 1;
      // the second row of an odd ny's last pair is zero; its (clamped)
      // value is loaded anyway, so both rows' loads go out together
      const float a0 = src.value(comp, x, y0, z, d);
      const float a1r = src.value(comp, x, y1 < ny ? y1 : y0, z, d);
      const float a1 = y1 < ny ? a1r : 0.f;
      A[b * nx + x] = make_float2(a0, a1);
    }
    __syncthreads();
    const float2 *R = fft_lines<-1>(A, B, pb, nx, p.ax);
    // two real rows from one complex transform:
    // X0[k] = (Z[k] + conj Z[n-k]) / 2,  X1[k] = (Z[k] - conj Z[n-k]) / 2i
    for (int t = threadIdx.x; t < pb * nxh; t += blockDim.x) {
      const int b = t / nxh, k = t - b * nxh;
      const float2 Z = R[b * nx + k];
      const float2 Zm = R[b * nx + (k == 0 ? 0 : nx - k)];
      const int y0 = 2 * (p0 + b), y1 = y0 + 1;
      C[y0 * nxh + k] = make_float2(0.5f * (Z.x + Zm.x), 0.5f * (Z.y - Zm.y));
      if (y1 < ny) C[y1 * nxh + k] = make_float2(0.5f * (Z.y + Zm.y), -0.5f * (Z.x - Zm.x));
    }
    __syncthreads();
  }
  float2 *out = p.spec + ((long)comp * d.nz + z) * ny * nxh;
  for (int k0 = 0; k0 < nxh; k0 += Q) {
    const int qb = min(Q, nxh - k0);
    for (int t = threadIdx.x; t < qb * ny; t += blockDim.x) {
      const int y = t / qb, q = t - y * qb;
      A[q * ny + y] = C[y * nxh + k0 + q];
    }
    __syncthreads();
    const float2 *R = fft_lines<-1>(A, B, qb, ny, p.ay);
    for (int t = threadIdx.x; t < qb * ny; t += blockDim.x) {
      const int y = t / qb, q = t - y * qb;
      out[(long)y * nxh + k0 + q] = R[q * ny + y];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_fft_z_solve(FluidPlan p, int inverse) {
  extern __shared__ float2 sm[];
  const int nz = p.d.nz, nxh = p.nxh;
  const int K = p.zcols_per_cta;
  const long ncols = (long)p.d.ny * nxh;
  const long j0 = (long)blockIdx.x * K;
  const int kb = (int)min((long)K, ncols - j0);
  const long plane = ncols;  // complex elements per z-plane of one component
  float2 *A = sm;
  float2 *B = A + 3 * K * nz;
  for (int t = threadIdx.x; t < 3 * kb * nz; t += blockDim.x) {
    const int q = t % kb;
    const int r = t / kb;  // r = c*nz + kz
    const int c = r / nz, kz = r - c * nz;
    A[(c * K + q) * nz + kz] = p.spec[((long)c * nz + kz) * plane + j0 + q];
  }
  __syncthreads();
  // lines: c*K + q for c in 0..2, q in 0..kb-1 (unused q in [kb,K) skipped via ld stride)
  float2 *R = fft_lines<-1>(A, B, 3 * K, nz, p.az);
  float2 *W = (R == A) ? B : A;
  const float *cwx = p.lut, *swx = cwx + p.d.nx, *cwy = swx + p.d.nx, *swy = cwy + p.d.ny,
              *cwz = swy + p.d.ny, *swz = cwz + nz;
  const float invN = 1.0f / (float)p.d.n();
  for (int t = threadIdx.x; t < kb * nz; t += blockDim.x) {
    const int q = t % kb, kz = t / kb;
    const long j = j0 + q;
    const int ky = (int)(j / nxh), kx = (int)(j - (long)ky * nxh);
    const float cx = __ldg(cwx + kx), cy = __ldg(cwy + ky), cz = __ldg(cwz + kz);
    const float sx = __ldg(swx + kx), sy = __ldg(swy + ky), sz = __ldg(swz + kz);
    const float lambda = -p.alpha * (cx + cy + cz) + p.gamma;
    const float L00 = lambda - p.beta * cx, L11 = lambda - p.beta * cy, L22 = lambda - p.beta * cz;
    const float L10 = p.beta * sx * sy, L20 = p.beta * sx * sz, L21 = p.beta * sy * sz;
    float2 b0 = R[(0 * K + q) * nz + kz], b1 = R[(1 * K + q) * nz + kz], b2 = R[(2 * K + q) * nz + kz];
    b0.x *= invN; b0.y *= invN; b1.x *= invN; b1.y *= invN; b2.x *= invN; b2.y *= invN;
    float2 o0, o1, o2;
    if (inverse) {
      // Cholesky L = G G^T, then G y = b, G^T x = y (real matrix, complex rhs)
      const float G00 = sqrtf(L00);
      const float G10 = L10 / G00, G20 = L20 / G00;
      const float G11 = sqrtf(L11 - G10 * G10);
      const float G21 = (L21 - G20 * G10) / G11;
      const float G22 = sqrtf(L22 - (G20 * G20 + G21 * G21));
      float2 y0, y1, y2;
      y0.x = b0.x / G00;                              y0.y = b0.y / G00;
      y1.x = (b1.x - G10 * y0.x) / G11;               y1.y = (b1.y - G10 * y0.y) / G11;
      y2.x = (b2.x - G20 * y0.x - G21 * y1.x) / G22;  y2.y = (b2.y - G20 * y0.y - G21 * y1.y) / G22;
      o2.x = y2.x / G22;                              o2.y = y2.y / G22;
      o1.x = (y1.x - G21 * o2.x) / G11;               o1.y = (y1.y - G21 * o2.y) / G11;
      o0.x = (y0.x - G10 * o1.x - G20 * o2.x) / G00;  o0.y = (y0.y - G10 * o1.y - G20 * o2.y) / G00;
    } else {
      o0.x = L00 * b0.x + L10 * b1.x + L20 * b2.x;  o0.y = L00 * b0.y + L10 * b1.y + L20 * b2.y;
      o1.x = L10 * b0.x + L11 * b1.x + L21 * b2.x;  o1.y = L10 * b0.y + L11 * b1.y + L21 * b2.y;
      o2.x = L20 * b0.x + L21 * b1.x + L22 * b2.x;  o2.y = L20 * b0.y + L21 * b1.y + L22 * b2.y;
    }
    W[(0 * K + q) * nz + kz] = o0;
    W[(1 * K + q) * nz + kz] = o1;
    W[(2 * K + q) * nz + kz] = o2;
  }
  __syncthreads();
  const float2 *V = fft_lines<+1>(W, R, 3 * K, nz, p.az);
  for (int t = threadIdx.x; t < 3 * kb * nz; t += blockDim.x) {
    const int q = t % kb;
    const int r = t / kb;
    const int c = r / nz, kz = r - c * nz;
    p.spec[((long)c * nz + kz) * plane + j0 + q] = V[(c * K + q) * nz + kz];
  }
}

template <class Dst>
__global__ void __launch_bounds__(256) k_fft_xy_inv(FluidPlan p, Dst dst) {
  extern __shared__ float2 sm[];
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nxh = p.nxh;
  const int P = p.pairs_per_batch, Q = p.cols_per_batch;
  const int ws = max(P * nx, Q * ny);
  float2 *C = sm;
  float2 *A = C + ny * nxh;
  float2 *B = A + ws;
  const float2 *in = p.spec + ((long)comp * d.nz + z) * ny * nxh;
  for (int k0 = 0; k0 < nxh; k0 += Q) {
    const int qb = min(Q, nxh - k0);
    for (int t = threadIdx.x; t < qb * ny; t += blockDim.x) {
      const int y = t / qb, q = t - y * qb;
      A[q * ny + y] = in[(long)y * nxh + k0 + q];
    }
    __syncthreads();
    const float2 *R = fft_lines<+1>(A, B, qb, ny, p.ay);
    for (int t = threadIdx.x; t < qb * ny; t += blockDim.x) {
      const int y = t / qb, q = t - y * qb;
      C[y * nxh + k0 + q] = R[q * ny + y];
    }
    __syncthreads();
  }
  const int npairs = (ny + 1) >> 1;
  const bool even = (nx & 1) == 0;
  const auto out = dst.bind(comp);
  for (int p0 = 0; p0 < npairs; p0 += P) {
    const int pb = min(P, npairs - p0);
    // Z[k] = X0[k] + i X1[k] over the Hermitian completion; the imaginary
    // parts of the DC (and even-n Nyquist) terms are dropped, as c2r does.
    for (int t = threadIdx.x; t < pb * nx; t += blockDim.x) {
      const int b = t / nx, k = t - b * nx;
      const int y0 = 2 * (p0 + b), y1 = y0 + 1;
      const bool upper = k >= nxh;
      const int kk = upper ? nx - k : k;
      float2 X0 = C[y0 * nxh + kk];
      float2 X1 = (y1 < ny) ? C[y1 * nxh + kk] : make_float2(0.f, 0.f);
      if (kk == 0 || (even && kk == nx / 2)) { X0.y = 0.f; X1.y = 0.f; }
      if (upper) { X0.y = -X0.y; X1.y = -X1.y; }
      A[b * nx + k] = make_float2(X0.x - X1.y, X0.y + X1.x);
    }
    __syncthreads();
    const float2 *R = fft_lines<+1>(A, B, pb, nx, p.ax);
    for (int t = threadIdx.x; t < pb * nx; t += blockDim.x) {
      const int b = t / nx, x = t - b * nx;
      const int y0 = 2 * (p0 + b), y1 = y0 + 1;
      const float2 v = R[b * nx + x];
      out.store(d.idx(x, y0, z), v.x);
      if (y1 < ny) out.store(d.idx(x, y1, z), v.y);
    }
    __syncthreads();
  }
}

// ---- the split path: slabs larger than one CTA's shared memory ------------
// The same line transforms as k_fft_xy_fwd / k_fft_xy_inv (same batches,
// same fft_lines calls, so the same values), but the x and y passes are
// separate kernels and the half spectrum between them lives in HBM: an x
// pass CTA owns a batch of row pairs of one (z, component), a y pass CTA a
// batch of kx columns.

// x pass: producer -> R2C along x -> half-spectrum rows in the spectrum
template <class Src>
__global__ void __launch_bounds__(256) k_fft_x_fwd(FluidPlan p, Src src) {
  extern __shared__ float2 sm[];
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nxh = p.nxh;
  const int P = p.pairs_per_batch;
  float2 *A = sm;
  float2 *B = A + P * nx;
  const int npairs = (ny + 1) >> 1;
  const int p0 = blockIdx.z * P;
  const int pb = min(P, npairs - p0);
  for (int t = threadIdx.x; t < pb * nx; t += blockDim.x) {
    const int b = t / nx, x = t - b * nx;
    const int y0 = 2 * (p0 + b), y1 = y0 + 1;
    // as in k_fft_xy_fwd: both rows' loads go out together
    const float a0 = src.value(comp, x, y0, z, d);
    const float a1r = src.value(comp, x, y1 < ny ? y1 : y0, z, d);
    const float a1 = y1 < ny ? a1r : 0.f;
    A[b * nx + x] = make_float2(a0, a1);
  }
  __syncthreads();
  const float2 *R = fft_lines<-1>(A, B, pb, nx, p.ax);
  float2 *C = p.spec + ((long)comp * d.nz + z) * ny * nxh;
  for (int t = threadIdx.x; t < pb * nxh; t += blockDim.x) {
    const int b = t / nxh, k = t - b * nxh;
    const float2 Z = R[b * nx + k];
    const float2 Zm = R[b * nx + (k == 0 ? 0 : nx - k)];
    const int y0 = 2 * (p0 + b), y1 = y0 + 1;
    C[(long)y0 * nxh + k] = make_float2(0.5f * (Z.x + Zm.x), 0.5f * (Z.y - Zm.y));
    if (y1 < ny) C[(long)y1 * nxh + k] = make_float2(0.5f * (Z.y + Zm.y), -0.5f * (Z.x - Zm.x));
  }
}

// y pass, in place in the spectrum: a batch of kx columns of one (z, component)
template <int SIGN>
__global__ void __launch_bounds__(256) k_fft_y(FluidPlan p) {
  extern __shared__ float2 sm[];
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  const int ny = d.ny, nxh = p.nxh;
  const int Q = p.cols_per_batch;
  float2 *A = sm;
  float2 *B = A + Q * ny;
  const int k0 = blockIdx.z * Q;
  const int qb = min(Q, nxh - k0);
  float2 *C = p.spec + ((long)comp * d.nz + z) * ny * nxh;
  for (int t = threadIdx.x; t < qb * ny; t += blockDim.x) {
    const int y = t / qb, q = t - y * qb;
    A[q * ny + y] = C[(long)y * nxh + k0 + q];
  }
  __syncthreads();
  const float2 *R = fft_lines<SIGN>(A, B, qb, ny, p.ay);
  for (int t = threadIdx.x; t < qb * ny; t += blockDim.x) {
    const int y = t / qb, q = t - y * qb;
    C[(long)y * nxh + k0 + q] = R[q * ny + y];
  }
}

// x pass of the inverse: half-spectrum rows -> C2R along x -> consumer
template <class Dst>
__global__ void __launch_bounds__(256) k_fft_x_inv(FluidPlan p, Dst dst) {
  extern __shared__ float2 sm[];
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nxh = p.nxh;
  const int P = p.pairs_per_batch;
  float2 *A = sm;
  float2 *B = A + P * nx;
  const int npairs = (ny + 1) >> 1;
  const int p0 = blockIdx.z * P;
  const int pb = min(P, npairs - p0);
  const bool even = (nx & 1) == 0;
  const float2 *C = p.spec + ((long)comp * d.nz + z) * ny * nxh;
  for (int t = threadIdx.x; t < pb * nx; t += blockDim.x) {
    const int b = t / nx, k = t - b * nx;
    const int y0 = 2 * (p0 + b), y1 = y0 + 1;
    const bool upper = k >= nxh;
    const int kk = upper ? nx - k : k;
    float2 X0 = C[(long)y0 * nxh + kk];
    float2 X1 = (y1 < ny) ? C[(long)y1 * nxh + kk] : make_float2(0.f, 0.f);
    if (kk == 0 || (even && kk == nx / 2)) { X0.y = 0.f; X1.y = 0.f; }
    if (upper) { X0.y = -X0.y; X1.y = -X1.y; }
    A[b * nx + k] = make_float2(X0.x - X1.y, X0.y + X1.x);
  }
  __syncthreads();
  const float2 *R = fft_lines<+1>(A, B, pb, nx, p.ax);
  const auto out = dst.bind(comp);
  for (int t = threadIdx.x; t < pb * nx; t += blockDim.x) {
    const int b = t / nx, x = t - b * nx;
    const int y0 = 2 * (p0 + b), y1 = y0 + 1;
    const float2 v = R[b * nx + x];
    out.store(d.idx(x, y0, z), v.x);
    if (y1 < ny) out.store(d.idx(x, y1, z), v.y);
  }
}

template <class Src>
cudaError_t split_forward(const FluidPlan &p, const Src &src, cudaStream_t s) {
  const int npairs = (p.d.ny + 1) / 2;
  const int bx = (npairs + p.pairs_per_batch - 1) / p.pairs_per_batch;
  const int by = (p.nxh + p.cols_per_batch - 1) / p.cols_per_batch;
  k_fft_x_fwd<Src><<<dim3(p.d.nz, 3, bx), 256, p.smem_x, s>>>(p, src);
  k_fft_y<-1><<<dim3(p.d.nz, 3, by), 256, p.smem_y, s>>>(p);
  return cudaGetLastError();
}

template <class Dst>
cudaError_t split_inverse(const FluidPlan &p, const Dst &dst, cudaStream_t s) {
  const int npairs = (p.d.ny + 1) / 2;
  const int bx = (npairs + p.pairs_per_batch - 1) / p.pairs_per_batch;
  const int by = (p.nxh + p.cols_per_batch - 1) / p.cols_per_batch;
  k_fft_y<+1><<<dim3(p.d.nz, 3, by), 256, p.smem_y, s>>>(p);
  k_fft_x_inv<Dst><<<dim3(p.d.nz, 3, bx), 256, p.smem_x, s>>>(p, dst);
  return cudaGetLastError();
}

// TMA descriptor of the spectrum for the z-pass: a 3D float tensor
// {2*ny*nxh, nz, 3} read and written in boxes {2*Kq, nz, 1} = one row per
// kz of 16 columns (128 bytes, 128-byte swizzle) or 8 (64 bytes, 64-byte
// swizzle) in shared memory
bool encode_spec_map(FluidPlan *p) {
  const PFN_cuTensorMapEncodeTiled encode = tensor_map_encoder();
  if (!encode) return false;
  const cuuint64_t ncols = (cuuint64_t)p->d.ny * p->nxh;
  const cuuint64_t dims[3] = {2 * ncols, (cuuint64_t)p->d.nz, 3};
  const cuuint64_t strides[2] = {2 * ncols * sizeof(float), 2 * ncols * sizeof(float) * p->d.nz};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * p->fast_kq), (cuuint32_t)p->d.nz, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const size_t row = box[0] * sizeof(float);
  if ((row != 128 && row != 64) || box[1] > 256 || strides[0] % 16) return false;
  return encode(&p->spec_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, p->spec, dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE,
                row == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The register path's z-pass tile width (16 or 8 columns) by timing: after
// one untimed launch, three alternating L^-1 / L launches (the spectrum
// keeps its scale) of each on a zeroed spectrum; the faster is kept per
// (grid, device) for the process. The arithmetic of a column does not
// depend on the width.
std::mutex g_zq_mu;
std::map<std::tuple<int, int, int, int>, int> g_zq;

void tune_z_cols(FluidPlan *p) {
  const auto key = std::make_tuple(p->d.nx, p->d.ny, p->d.nz, p->device);
  {
    std::lock_guard<std::mutex> lock(g_zq_mu);
    auto it = g_zq.find(key);
    if (it != g_zq.end()) {
      p->fast_kq = it->second;
      p->fast_tma = encode_spec_map(p);
      return;
    }
  }
  const size_t bytes = sizeof(float2) * 3 * (size_t)p->d.nz * p->d.ny * p->nxh;
  if (cudaMemset(p->spec, 0, bytes) != cudaSuccess) return;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return;
  }
  float best = 1e30f;
  int pick = 16;
  for (int q : {16, 8}) {
    p->fast_kq = q;
    p->fast_tma = encode_spec_map(p);
    fast_z_solve(*p, 1, 0);
    cudaEventRecord(e0, 0);
    for (int r = 0; r < 3; ++r) fast_z_solve(*p, r & 1, 0);
    cudaEventRecord(e1, 0);
    float ms = 0.f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      break;
    if (ms < best) {
      best = ms;
      pick = q;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  p->fast_kq = pick;
  p->fast_tma = encode_spec_map(p);
  if (cudaGetLastError() != cudaSuccess) return;
  std::lock_guard<std::mutex> lock(g_zq_mu);
  g_zq[key] = pick;
}

// The shared-memory limit is an attribute of the kernel, shared by every
// plan on the device: only ever raise it, so a plan created later with a
// smaller footprint cannot invalidate the launches of a larger one.
std::mutex g_smem_mu;
std::map<std::pair<const void *, int>, size_t> g_smem;

template <class K>
cudaError_t set_smem(K kernel, size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_smem_mu);
  size_t &cur = g_smem[{reinterpret_cast<const void *>(kernel), dev}];
  if (bytes <= cur) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

// Shapes of the shared-memory (any-size) path: x-line pairs and y-columns per
// batch of the xy kernels, (ky,kx) columns per CTA of the z kernel, and the
// shared memory they need.
void generic_shapes(FluidPlan *p, int P, int Q, int K) {
  const int nx = p->d.nx, ny = p->d.ny, nz = p->d.nz;
  p->pairs_per_batch = P;
  p->cols_per_batch = Q;
  p->zcols_per_cta = K;
  const size_t ws = std::max((size_t)P * nx, (size_t)Q * ny);
  p->smem_xy = sizeof(float2) * ((size_t)ny * p->nxh + 2 * ws);
  p->smem_z = sizeof(float2) * (size_t)(2 * 3 * K * nz);
  p->smem_x = sizeof(float2) * 2 * (size_t)P * nx;
  p->smem_y = sizeof(float2) * 2 * (size_t)Q * ny;
}

// whether the plan's shapes fit: the fused xy kernels' slab, or (split) the
// x and y passes' batch buffers, and the z pass
bool generic_fits(const FluidPlan &p, size_t maxsm) {
  const bool xy = p.split ? (p.smem_x <= maxsm && p.smem_y <= maxsm) : p.smem_xy <= maxsm;
  return xy && p.smem_z <= maxsm;
}

cudaError_t generic_configure(const FluidPlan &p) {
  cudaError_t e;
  if (p.split) {
    if ((e = set_smem(k_fft_x_fwd<SrcField>, p.smem_x)) != cudaSuccess) return e;
    if ((e = set_smem(k_fft_x_fwd<SrcForce>, p.smem_x)) != cudaSuccess) return e;
    if ((e = set_smem(k_fft_x_inv<DstField>, p.smem_x)) != cudaSuccess) return e;
    if ((e = set_smem(k_fft_x_inv<DstAxpby>, p.smem_x)) != cudaSuccess) return e;
    if ((e = set_smem(k_fft_x_inv<DstNeg>, p.smem_x)) != cudaSuccess) return e;
    if ((e = set_smem(k_fft_y<-1>, p.smem_y)) != cudaSuccess) return e;
    if ((e = set_smem(k_fft_y<+1>, p.smem_y)) != cudaSuccess) return e;
    return set_smem(k_fft_z_solve, p.smem_z);
  }
  if ((e = set_smem(k_fft_xy_fwd<SrcField>, p.smem_xy)) != cudaSuccess) return e;
  if ((e = set_smem(k_fft_xy_fwd<SrcForce>, p.smem_xy)) != cudaSuccess) return e;
  if ((e = set_smem(k_fft_xy_inv<DstField>, p.smem_xy)) != cudaSuccess) return e;
  if ((e = set_smem(k_fft_xy_inv<DstAxpby>, p.smem_xy)) != cudaSuccess) return e;
  if ((e = set_smem(k_fft_xy_inv<DstNeg>, p.smem_xy)) != cudaSuccess) return e;
  return set_smem(k_fft_z_solve, p.smem_z);
}

// autotuned shapes per (grid, device), kept for the life of the process
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, std::tuple<int, int, int>> g_tuned;

}  // namespace

int fluid_get_shapes(const FluidPlan &p, int *P, int *Q, int *K) {
  *P = p.fast ? 0 : p.pairs_per_batch;
  *Q = p.fast ? 0 : p.cols_per_batch;
  *K = p.fast ? p.fast_kq : p.zcols_per_cta;
  return p.fast ? 0 : 1;
}

cudaError_t fluid_set_shapes(FluidPlan *p, int P, int Q, int K) {
  const int npairs = (p->d.ny + 1) / 2;
  if (p->fast) {
    // the register path: only the z-pass tile width, 16 or 8 columns
    if (P != 0 || Q != 0 || (K != 16 && K != 8)) return cudaErrorInvalidValue;
    p->fast_kq = K;
    p->fast_tma = encode_spec_map(p);
    return cudaSuccess;
  }
  if (P < 1 || P > npairs || Q < 1 || Q > p->nxh || K < 1 || K > 64) return cudaErrorInvalidValue;
  FluidPlan t = *p;
  generic_shapes(&t, P, Q, K);
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device);
  if (!generic_fits(t, (size_t)maxsm)) return cudaErrorInvalidValue;
  const cudaError_t e = generic_configure(t);
  if (e == cudaSuccess) *p = t;
  return e;
}

// The shared-memory path's autotuner: every combination of half, the
// heuristic and twice the heuristic line pairs and columns per batch is
// timed on the forward + inverse xy pass, then 2..32 columns per z CTA on
// the z pass (alternating L^-1 and L so the spectrum keeps its scale), each
// the mean of three launches after one untimed, on a zero field (the
// arithmetic is the same for every shape; only the distribution of lines
// over CTAs changes). The choice is kept per grid and device.
cudaError_t fluid_autotune(FluidPlan *p, cudaStream_t s) {
  if (p->fast) return cudaSuccess;
  const auto key = std::make_tuple(p->d.nx, p->d.ny, p->d.nz, p->device);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end())
      return fluid_set_shapes(p, std::get<0>(it->second), std::get<1>(it->second),
                              std::get<2>(it->second));
  }
  const long n = p->d.n();
  float *f = nullptr;
  cudaError_t e = cudaMalloc(&f, sizeof(float) * 3 * n);
  if (e != cudaSuccess) {  // no room for the tuning field: keep the heuristic shapes
    cudaGetLastError();
    return cudaSuccess;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto timed = [&](auto &&fn, float *ms) -> cudaError_t {
    cudaError_t r = fn();
    if (r != cudaSuccess) return r;
    cudaEventRecord(e0, s);
    for (int i = 0; i < 3 && r == cudaSuccess; ++i) r = fn();
    cudaEventRecord(e1, s);
    if (r == cudaSuccess) r = cudaEventSynchronize(e1);
    if (r == cudaSuccess) r = cudaEventElapsedTime(ms, e0, e1);
    return r;
  };
  float *c[3] = {f, f + n, f + 2 * n};
  const int P0 = p->pairs_per_batch, Q0 = p->cols_per_batch, K0 = p->zcols_per_cta;
  int bestP = P0, bestQ = Q0, bestK = K0;
  float best = 1e30f;
  if ((e = cudaMemsetAsync(f, 0, sizeof(float) * 3 * n, s)) == cudaSuccess) {
    for (int P : {P0 / 2, P0, 2 * P0})
      for (int Q : {Q0 / 2, Q0, 2 * Q0}) {
        if (fluid_set_shapes(p, P, Q, K0) != cudaSuccess) continue;
        float ms = 0.f;
        if ((e = timed([&]() {
               cudaError_t r = fluid_forward_field(*p, c[0], c[1], c[2], s);
               return r == cudaSuccess ? fluid_inverse_store(*p, c[0], c[1], c[2], s) : r;
             }, &ms)) != cudaSuccess)
          break;
        if (ms < best) {
          best = ms;
          bestP = P;
          bestQ = Q;
        }
      }
  }
  if (e == cudaSuccess) {
    best = 1e30f;
    int flip = 0;
    for (int K : {2, 4, 8, 16, 32}) {
      if (fluid_set_shapes(p, bestP, bestQ, K) != cudaSuccess) continue;
      float ms = 0.f;
      if ((e = timed([&]() { return fluid_solve(*p, (flip++ & 1) ? 0 : 1, s); }, &ms)) !=
          cudaSuccess)
        break;
      if (ms < best) {
        best = ms;
        bestK = K;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(f);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[key] = std::make_tuple(bestP, bestQ, bestK);
  }
  return fluid_set_shapes(p, bestP, bestQ, bestK);
}

int fluid_plan_create(FluidPlan *p, int nx, int ny, int nz, double spx, double spy, double spz,
                      float alpha, float beta, float gamma) {
  std::memset(p, 0, sizeof(*p));
  if (nx < 2 || ny < 2 || nz < 2 || nx > 512 || ny > 512 || nz > 512) return 1;
  p->d = Dims{nx, ny, nz};
  p->sp = Spacing{spx, spy, spz};
  p->alpha = alpha;
  p->beta = beta;
  p->gamma = gamma;
  p->nxh = nx / 2 + 1;
  if (!factorize(nx, p->ax) || !factorize(ny, p->ay) || !factorize(nz, p->az)) return 1;
  const int npairs = (ny + 1) / 2;
  generic_shapes(p, std::max(1, std::min(npairs, (2048 + nx - 1) / nx)),
                 std::max(1, std::min(p->nxh, (2048 + ny - 1) / ny)),
                 std::max(1, std::min(16, 3072 / (3 * nz))));
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  p->device = dev;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (fast_supported(nx) && fast_supported(ny) && fast_supported(nz)) {
    p->fast_kq = fast_z_cols();
    p->fast_smem_xy = fast_xy_smem(nx, ny);
    p->fast_smem_z = fast_z_smem(nz, 16);
    p->fast = p->fast_smem_xy <= (size_t)maxsm && p->fast_smem_z <= (size_t)maxsm;
  }
  // a slab whose half spectrum does not fit one CTA: the split x / y passes
  if (!p->fast && p->smem_xy > (size_t)maxsm) p->split = 1;
  if (!p->fast && !generic_fits(*p, (size_t)maxsm)) return 2;

  std::vector<float2> tw;
  fill_twiddles(nx, tw);
  fill_twiddles(ny, tw);
  fill_twiddles(nz, tw);
  std::vector<float> lut;
  fill_lut(nx, spx, lut);
  fill_lut(ny, spy, lut);
  fill_lut(nz, spz, lut);
  if (cudaMalloc(&p->tw, tw.size() * sizeof(float2)) != cudaSuccess) return 3;
  if (cudaMalloc(&p->lut, lut.size() * sizeof(float)) != cudaSuccess) return 3;
  if (cudaMalloc(&p->spec, sizeof(float2) * 3 * (size_t)nz * ny * p->nxh) != cudaSuccess) return 3;
  if (cudaMalloc(&p->status, sizeof(int)) != cudaSuccess) return 3;
  cudaMemset(p->status, 0, sizeof(int));
  cudaMemcpy(p->tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice);
  cudaMemcpy(p->lut, lut.data(), lut.size() * sizeof(float), cudaMemcpyHostToDevice);
  p->ax.tw = p->tw;
  p->ay.tw = p->tw + nx;
  p->az.tw = p->tw + nx + ny;
  if (generic_configure(*p) != cudaSuccess) return 4;
  if (p->fast) p->fast_tma = encode_spec_map(p);
  if (p->fast && fast_configure(*p) != cudaSuccess) return 4;
  if (p->fast) tune_z_cols(p);
  if (!p->fast && fluid_autotune(p, 0) != cudaSuccess) return 4;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

namespace {

// The timeout path of the transform kernels, run on purpose: nothing ever
// arrives on this barrier, so every thread's bounded wait gives up after
// `polls` polls, the status word records it, and the CTA leaves together
// as a transform CTA does when its slab never lands. Nothing is in flight
// on the barrier when the CTA exits.
__global__ void k_wait_selftest(int *status, int polls) {
  __shared__ __align__(8) uint64_t mbar;
  if (threadIdx.x == 0) mbar_init(&mbar, 1);
  __syncthreads();
  const bool ok = mbar_wait(&mbar, 0, status, polls);
  (void)__syncthreads_or(!ok);
}

}  // namespace

cudaError_t fluid_wait_selftest(const FluidPlan &p, int polls, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(p.status, polls);
  return cudaGetLastError();
}

cudaError_t fluid_take_status(FluidPlan *p, int *timed_out, cudaStream_t s) {
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, p->status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  *timed_out = v == kStatusWaitTimeout ? 1 : 0;
  return v ? cudaMemsetAsync(p->status, 0, sizeof(int), s) : cudaSuccess;
}

void fluid_plan_destroy(FluidPlan *p) {
  if (p->tw) cudaFree(p->tw);
  if (p->lut) cudaFree(p->lut);
  if (p->spec) cudaFree(p->spec);
  if (p->status) cudaFree(p->status);
  std::memset(p, 0, sizeof(*p));
}

cudaError_t fluid_forward_field(const FluidPlan &p, const float *fx, const float *fy,
                                const float *fz, cudaStream_t s) {
  SrcField src{{fx, fy, fz}};
  if (p.fast) return fast_xy_forward(p, src, s);
  if (p.split) return split_forward(p, src, s);
  k_fft_xy_fwd<SrcField><<<dim3(p.d.nz, 3), 256, p.smem_xy, s>>>(p, src);
  return cudaGetLastError();
}

cudaError_t fluid_forward_force(const FluidPlan &p, const float *G, const float *A, int diff,
                                cudaStream_t s) {
  const SrcForce src = make_force(G, A, diff, p.sp);
  if (p.fast) return fast_xy_forward(p, src, s);
  if (p.split) return split_forward(p, src, s);
  k_fft_xy_fwd<SrcForce><<<dim3(p.d.nz, 3), 256, p.smem_xy, s>>>(p, src);
  return cudaGetLastError();
}

cudaError_t fluid_forward_force_jac(const FluidPlan &p, const float *G, const float *A,
                                    const float *B, cudaStream_t s) {
  const SrcForce src = make_force(G, A, 2, p.sp, B);
  if (p.fast) return fast_xy_forward(p, src, s);
  if (p.split) return split_forward(p, src, s);
  k_fft_xy_fwd<SrcForce><<<dim3(p.d.nz, 3), 256, p.smem_xy, s>>>(p, src);
  return cudaGetLastError();
}

cudaError_t fluid_solve(const FluidPlan &p, int inverse, cudaStream_t s) {
  if (p.fast) return fast_z_solve(p, inverse, s);
  const long ncols = (long)p.d.ny * p.nxh;
  const int grid = (int)((ncols + p.zcols_per_cta - 1) / p.zcols_per_cta);
  k_fft_z_solve<<<grid, 256, p.smem_z, s>>>(p, inverse);
  return cudaGetLastError();
}

cudaError_t fluid_inverse_store(const FluidPlan &p, float *ox, float *oy, float *oz,
                                cudaStream_t s) {
  DstField dst{{ox, oy, oz}};
  if (p.fast) return fast_xy_inverse(p, dst, s);
  if (p.split) return split_inverse(p, dst, s);
  k_fft_xy_inv<DstField><<<dim3(p.d.nz, 3), 256, p.smem_xy, s>>>(p, dst);
  return cudaGetLastError();
}

cudaError_t fluid_inverse_compose(const FluidPlan &p, const ComposeArgs &a, cudaStream_t s) {
  if (!p.fast) return cudaErrorNotSupported;
  return fast_xy_inverse_compose(p, a, s);
}

cudaError_t fluid_inverse_store_neg(const FluidPlan &p, float *ox, float *oy, float *oz,
                                    cudaStream_t s) {
  DstNeg dst{{ox, oy, oz}};
  if (p.fast) return fast_xy_inverse(p, dst, s);
  if (p.split) return split_inverse(p, dst, s);
  k_fft_xy_inv<DstNeg><<<dim3(p.d.nz, 3), 256, p.smem_xy, s>>>(p, dst);
  return cudaGetLastError();
}

cudaError_t fluid_inverse_axpby(const FluidPlan &p, float *vx, float *vy, float *vz,
                                const float *step, float sigma, cudaStream_t s) {
  DstAxpby dst{{vx, vy, vz}, step, sigma};
  if (p.fast) return fast_xy_inverse(p, dst, s);
  if (p.split) return split_inverse(p, dst, s);
  k_fft_xy_inv<DstAxpby><<<dim3(p.d.nz, 3), 256, p.smem_xy, s>>>(p, dst);
  return cudaGetLastError();
}

}  // namespace aw
