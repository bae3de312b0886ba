/*
 * sp_sf.cu -- structure factor of a device-resident field (post-processing at
 * save points, no counterpart on the step path).
 *
 * SymPhas's SF collector (dataprocesses/datasf.h:137-245) thresholds the field
 * (1 where the value is positive, else 0), takes its DFT, scales |F(k)|^2 by
 * 1 / (number of sites) and averages it radially
 * (datatypes/inc/datalib.h:1120-1330 with lib/src/spslib.cpp:32-200): the
 * averaging classes are the wave vectors whose absolute integer components
 * agree up to order, and the classes are ordered by sqrt(i^2 + j^2 + k^2).
 * Here the field is gathered from its padded layout on the device, transformed
 * with an FP64 real-to-complex FFT (cuFFT), and every point of the half
 * spectrum is added to its class with its multiplicity (2 for the points
 * whose conjugate partner is not stored, 1 otherwise); the class table is
 * built once per handle on the host.
 */
#include <cufft.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <tuple>

#include "sp_handle.h"

namespace sp {
namespace {

template <class T>
__global__ void k_sf_gather(const T* org, double* out, int n0, int n1, int n2, long long pitch,
                            long long plane, int threshold) {
  const long long total = (long long)n0 * n1 * n2;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const long long x = id % n0, y = (id / n0) % n1, z = id / ((long long)n0 * n1);
    const double v = double(org[z * plane + y * pitch + x]);
    out[id] = threshold ? (v > 0.0 ? 1.0 : 0.0) : v;
  }
}

// half spectrum (n2, n1, n0 / 2 + 1) -> class sums; map is indexed by the
// absolute wave-vector components (|kz| (n1/2+1) + |ky|) (n0/2+1) + |kx|
__global__ void k_sf_bin(const cufftDoubleComplex* F, int n0, int n1, int n2, const int* map,
                         double* sum, double* cnt) {
  const int hx = n0 / 2 + 1, hy = n1 / 2 + 1;
  const long long total = (long long)hx * n1 * n2;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int x = int(id % hx), y = int((id / hx) % n1), z = int(id / ((long long)hx * n1));
    const int ay = y <= n1 - y ? y : n1 - y, az = z <= n2 - z ? z : n2 - z;
    const double w = (x == 0 || (n0 % 2 == 0 && x == n0 / 2)) ? 1.0 : 2.0;
    const cufftDoubleComplex c = F[id];
    const int b = map[((long long)az * hy + ay) * hx + x];
    atomicAdd(&sum[b], w * (c.x * c.x + c.y * c.y));
    atomicAdd(&cnt[b], w);
  }
}

struct SfTable {
  std::vector<int> map;        // octant index -> class
  std::vector<double> radius;  // class -> sqrt(i^2 + j^2 + k^2)
};

// classes of the octant [0, n0/2] x [0, n1/2] x [0, n2/2]: sorted triples of
// absolute components, numbered in order of radius (ties by triple)
SfTable sf_table(const int n[3]) {
  const int hx = n[0] / 2 + 1, hy = n[1] / 2 + 1, hz = n[2] / 2 + 1;
  std::map<std::tuple<long long, int, int, int>, int> classes;
  std::vector<std::array<int, 3>> key((size_t)hx * hy * hz);
  for (int k = 0; k < hz; ++k)
    for (int j = 0; j < hy; ++j)
      for (int i = 0; i < hx; ++i) {
        std::array<int, 3> t{i, j, k};
        std::sort(t.begin(), t.end());
        key[((size_t)k * hy + j) * hx + i] = t;
        const long long r2 = (long long)i * i + (long long)j * j + (long long)k * k;
        classes.emplace(std::make_tuple(r2, t[0], t[1], t[2]), 0);
      }
  SfTable tab;
  std::map<std::array<int, 3>, int> id;
  tab.radius.reserve(classes.size());
  int c = 0;
  for (auto& kv : classes) {
    const auto& [r2, a, b, d] = kv.first;
    id[{a, b, d}] = c++;
    tab.radius.push_back(std::sqrt(double(r2)));
  }
  tab.map.resize(key.size());
  for (size_t q = 0; q < key.size(); ++q) tab.map[q] = id[key[q]];
  return tab;
}

}  // namespace
}  // namespace sp

extern "C" int sp_structure_factor(sp_handle* H, int inst, int field, int threshold,
                                   double* k_out, double* s_out, int* nbins) {
  if (!H || !nbins) return SP_EINVAL;
  if (inst < 0 || inst >= H->batch || field < 0 || field >= H->nf) {
    H->err = "instance or field index out of range";
    return SP_EINVAL;
  }
  const InstGeo& g = H->geo[inst];
  int n[3] = {g.n[0], g.n[1], H->dim == 3 ? g.n[2] : 1};
  const sp::SfTable tab = sp::sf_table(n);
  const int nb = int(tab.radius.size());
  if (!k_out || !s_out) {
    *nbins = nb;
    return SP_OK;
  }
  if (*nbins < nb) {
    H->err = "output arrays shorter than the number of classes";
    *nbins = nb;
    return SP_EINVAL;
  }
  const long long total = (long long)n[0] * n[1] * n[2];
  const long long half = (long long)(n[0] / 2 + 1) * n[1] * n[2];
  double* real = nullptr;
  cufftDoubleComplex* spec = nullptr;
  int* map = nullptr;
  double* acc = nullptr;
  cufftHandle plan = 0;
  bool planned = false;
  int rc = SP_OK;
  auto cuda = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == SP_OK) {
      H->err = std::string(what) + ": " + cudaGetErrorString(e);
      rc = e == cudaErrorMemoryAllocation ? SP_ENOMEM : SP_ECUDA;
    }
    return rc == SP_OK;
  };
  const int blocks = int(std::min<long long>(H->sms * 8LL, (total + 255) / 256));
  if (cuda(cudaMalloc(&real, sizeof(double) * total), "cudaMalloc") &&
      cuda(cudaMalloc(&spec, sizeof(cufftDoubleComplex) * half), "cudaMalloc") &&
      cuda(cudaMalloc(&map, sizeof(int) * tab.map.size()), "cudaMalloc") &&
      cuda(cudaMalloc(&acc, sizeof(double) * 2 * nb), "cudaMalloc") &&
      cuda(cudaMemcpyAsync(map, tab.map.data(), sizeof(int) * tab.map.size(),
                           cudaMemcpyHostToDevice, H->stream), "cudaMemcpyAsync") &&
      cuda(cudaMemsetAsync(acc, 0, sizeof(double) * 2 * nb, H->stream), "cudaMemsetAsync")) {
    const char* org = field_origin(H, H->cur, inst, field);
    if (H->esz == 4)
      sp::k_sf_gather<float><<<blocks, 256, 0, H->stream>>>(
          reinterpret_cast<const float*>(org), real, n[0], n[1], n[2], g.pitch, g.plane,
          threshold);
    else
      sp::k_sf_gather<double><<<blocks, 256, 0, H->stream>>>(
          reinterpret_cast<const double*>(org), real, n[0], n[1], n[2], g.pitch, g.plane,
          threshold);
    cuda(cudaGetLastError(), "gather");
    cufftResult fr = H->dim == 3 ? cufftPlan3d(&plan, n[2], n[1], n[0], CUFFT_D2Z)
                                 : cufftPlan2d(&plan, n[1], n[0], CUFFT_D2Z);
    planned = fr == CUFFT_SUCCESS;
    if (fr == CUFFT_SUCCESS) fr = cufftSetStream(plan, H->stream);
    if (fr == CUFFT_SUCCESS) fr = cufftExecD2Z(plan, real, spec);
    if (fr != CUFFT_SUCCESS && rc == SP_OK) {
      H->err = "cuFFT failed (cufftResult " + std::to_string(int(fr)) + ")";
      rc = SP_ECUDA;
    }
    if (rc == SP_OK) {
      const int bb = int(std::min<long long>(H->sms * 8LL, (half + 255) / 256));
      sp::k_sf_bin<<<bb, 256, 0, H->stream>>>(spec, n[0], n[1], n[2], map, acc, acc + nb);
      cuda(cudaGetLastError(), "binning");
    }
    std::vector<double> host(2 * (size_t)nb);
    if (rc == SP_OK &&
        cuda(cudaMemcpyAsync(host.data(), acc, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost,
                             H->stream), "cudaMemcpyAsync") &&
        cuda(cudaStreamSynchronize(H->stream), "cudaStreamSynchronize")) {
      for (int b = 0; b < nb; ++b) {
        k_out[b] = tab.radius[b];
        s_out[b] = host[nb + b] > 0 ? host[b] / host[nb + b] / double(total) : 0.0;
      }
      *nbins = nb;
    }
  }
  if (planned) cufftDestroy(plan);
  cudaFree(real);
  cudaFree(spec);
  cudaFree(map);
  cudaFree(acc);
  return rc;
}
