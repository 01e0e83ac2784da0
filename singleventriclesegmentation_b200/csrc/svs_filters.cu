// Pre- and post-filters of the flow path: the Gaussian pre-blur (svs/utils/flow_utils.py:94-112)
// and the 3x3x3 median post-filter (flow_utils.py:115-132), both on the device.
#include <cuda_runtime.h>

#include "svs_common.cuh"

namespace svs {
namespace {

constexpr int kMaxBlurTaps = 13 * 13 * 13;  // sigma up to 2.6 (kernel size int(5 sigma) made odd)

template <typename T>
struct BlurWeights {
  T w[kMaxBlurTaps];
};

// Zero-padded 3D correlation with a (2r+1)^3 kernel (F.conv3d, padding = r). Accumulates in
// the value type in (z, y, x) tap order.
template <typename T>
__global__ void blur_kernel(const T* __restrict__ in, int nz, int ny, int nx, int r,
                            const __grid_constant__ BlurWeights<T> W, T* __restrict__ out) {
  const int64_t n = (int64_t)nz * ny * nx;
  const int k = 2 * r + 1;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    T acc = T(0);
    for (int a = 0; a < k; ++a) {
      const int zz = z + a - r;
      if (zz < 0 || zz >= nz) continue;
      for (int b = 0; b < k; ++b) {
        const int yy = y + b - r;
        if (yy < 0 || yy >= ny) continue;
        const T* row = in + ((size_t)zz * ny + yy) * nx;
        const T* wr = W.w + (a * k + b) * k;
        for (int c = 0; c < k; ++c) {
          const int xx = x + c - r;
          if (xx >= 0 && xx < nx) acc = fma(wr[c], __ldg(row + xx), acc);
        }
      }
    }
    out[v] = acc;
  }
}

// Median of 27 by rank counting: the element with fewer than 14 smaller values and at least 14
// values not larger than it (exact with ties, no sorting network state).
template <typename T>
__device__ __forceinline__ T median27(const T (&w)[27]) {
  T med = w[0];
#pragma unroll 1
  for (int i = 0; i < 27; ++i) {
    int lt = 0, le = 0;
#pragma unroll
    for (int j = 0; j < 27; ++j) {
      lt += w[j] < w[i];
      le += w[j] <= w[i];
    }
    if (lt <= 13 && le > 13) med = w[i];
  }
  return med;
}

// ks^3 median of each component with scipy 'reflect' (== MIRROR fold) at the faces.
template <typename T>
__global__ void median3_kernel(const T* __restrict__ in, int nz, int ny, int nx, int C,
                               T* __restrict__ out) {
  const int64_t n = (int64_t)nz * ny * nx * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(t % C);
    const int64_t v = t / C;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    T w[27];
    int m = 0;
#pragma unroll
    for (int a = -1; a <= 1; ++a) {
      const int zz = fold(z + a, nz, SVS_BOUNDARY_MIRROR);
#pragma unroll
      for (int b = -1; b <= 1; ++b) {
        const int yy = fold(y + b, ny, SVS_BOUNDARY_MIRROR);
#pragma unroll
        for (int d = -1; d <= 1; ++d) {
          const int xx = fold(x + d, nx, SVS_BOUNDARY_MIRROR);
          w[m++] = __ldg(in + (((size_t)zz * ny + yy) * nx + xx) * C + c);
        }
      }
    }
    out[t] = median27(w);
  }
}

// Generic odd window (ks = 5 or 7): partial selection sort in local memory up to the median rank.
template <typename T>
__global__ void median_generic_kernel(const T* __restrict__ in, int nz, int ny, int nx, int C,
                                      int ks, T* __restrict__ out) {
  const int64_t n = (int64_t)nz * ny * nx * C;
  const int r = ks / 2, cnt = ks * ks * ks;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(t % C);
    const int64_t v = t / C;
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((int64_t)nx * ny));
    T w[343];
    int m = 0;
    for (int a = -r; a <= r; ++a)
      for (int b = -r; b <= r; ++b)
        for (int d = -r; d <= r; ++d)
          w[m++] = __ldg(in + (((size_t)fold(z + a, nz, SVS_BOUNDARY_MIRROR) * ny +
                                fold(y + b, ny, SVS_BOUNDARY_MIRROR)) * nx +
                               fold(x + d, nx, SVS_BOUNDARY_MIRROR)) * C + c);
    const int rank = cnt / 2;
    for (int i = 0; i <= rank; ++i) {
      int best = i;
      for (int j = i + 1; j < cnt; ++j)
        if (w[j] < w[best]) best = j;
      const T tmp = w[i]; w[i] = w[best]; w[best] = tmp;
    }
    out[t] = w[rank];
  }
}

unsigned grid_for(int64_t n, int threads) {
  const int64_t blocks = (n + threads - 1) / threads;
  return (unsigned)(blocks < 148 * 64 ? (blocks > 0 ? blocks : 1) : 148 * 64);
}

}  // namespace
}  // namespace svs

using namespace svs;

namespace svs {
namespace {

template <typename T>
svs_status gauss_blur3d(const char* nm, const T* in, int nz, int ny, int nx, const T* weights_host, int r, T* out,
                        cudaStream_t stream) {
  SVS_REQUIRE(in && out && weights_host, std::string(nm) + ": null pointer");
  SVS_REQUIRE(nz > 0 && ny > 0 && nx > 0, std::string(nm) + ": bad sizes");
  SVS_REQUIRE(r >= 0 && (2 * r + 1) * (2 * r + 1) * (2 * r + 1) <= kMaxBlurTaps,
              std::string(nm) + ": kernel radius out of range (max 6)");
  BlurWeights<T> W;
  const int k = 2 * r + 1;
  for (int i = 0; i < k * k * k; ++i) W.w[i] = weights_host[i];
  const int64_t n = (int64_t)nz * ny * nx;
  blur_kernel<T><<<grid_for(n, 256), 256, 0, stream>>>(in, nz, ny, nx, r, W, out);
  return check_launch(nm);
}

template <typename T>
svs_status median3d(const char* nm, const T* in, int nz, int ny, int nx, int C, int ks, T* out, cudaStream_t stream) {
  SVS_REQUIRE(in && out, std::string(nm) + ": null pointer");
  SVS_REQUIRE(nz > 0 && ny > 0 && nx > 0 && C > 0, std::string(nm) + ": bad sizes");
  SVS_REQUIRE(ks == 1 || ks == 3 || ks == 5 || ks == 7, std::string(nm) + ": kernel size must be 1, 3, 5 or 7");
  const int64_t n = (int64_t)nz * ny * nx * C;
  if (ks == 1) return check_cuda(cudaMemcpyAsync(out, in, n * sizeof(T), cudaMemcpyDeviceToDevice, stream), nm);
  if (ks == 3) median3_kernel<T><<<grid_for(n, 256), 256, 0, stream>>>(in, nz, ny, nx, C, out);
  else median_generic_kernel<T><<<grid_for(n, 128), 128, 0, stream>>>(in, nz, ny, nx, C, ks, out);
  return check_launch(nm);
}

}  // namespace
}  // namespace svs

extern "C" {

svs_status svs_gauss_blur3d(const float* in, int nz, int ny, int nx, const float* weights_host, int r, float* out,
                            svs_stream_t stream) {
  return gauss_blur3d<float>("svs_gauss_blur3d", in, nz, ny, nx, weights_host, r, out, stream);
}
svs_status svs_gauss_blur3d_f64(const double* in, int nz, int ny, int nx, const double* weights_host, int r,
                                double* out, svs_stream_t stream) {
  return gauss_blur3d<double>("svs_gauss_blur3d_f64", in, nz, ny, nx, weights_host, r, out, stream);
}
svs_status svs_median3d(const float* in, int nz, int ny, int nx, int C, int ks, float* out, svs_stream_t stream) {
  return median3d<float>("svs_median3d", in, nz, ny, nx, C, ks, out, stream);
}
svs_status svs_median3d_f64(const double* in, int nz, int ny, int nx, int C, int ks, double* out,
                            svs_stream_t stream) {
  return median3d<double>("svs_median3d_f64", in, nz, ny, nx, C, ks, out, stream);
}

}  // extern "C"
