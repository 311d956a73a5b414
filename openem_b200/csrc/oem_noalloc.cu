// Volume-weighted field sums without any device allocation.
//
// oem_plan_energy computes the float64 sums the early-termination criteria need
// (sum V|E|^2, sum V eps|E|^2, sum V|H|^2) with a per-block partial-sum buffer the plan
// allocates. Some callers cannot allocate device memory at the point where they need these
// sums: code that keeps its own fields in memory owned by another framework's pool (where a
// cudaMalloc outside the pool competes with it for the last free gigabytes and fragments it),
// and step loops that must not stall, since cudaMalloc and cudaFree can synchronise the whole
// device. oem_field_energy_noalloc serves them: the caller passes the six field arrays, the
// permittivity arrays and the grid spacings, and receives the three sums; the only device
// memory it touches besides those inputs is one file-scope scratch array, 581 KB on every GPU
// that loads this library, held until the process exits.
//
// Limits and sharing:
//   * nx + ny + nz must not exceed kMaxAxisCells (32768); larger grids get OEM_ERR_INVALID.
//   * The scratch array is shared by every call in the process. Each call overwrites the parts
//     it reads (block partials, totals, spacings) before reading them, so nothing needs to be
//     cleared between calls; but two calls whose work overlaps on the GPU (different streams,
//     or different host threads) race on it and return wrong sums.
//   * The first call on each device looks up the array's device address with
//     cudaGetSymbolAddress. With CUDA's lazy module loading (the default since CUDA 12) that
//     first lookup is also what loads this library's module onto the device, which can itself
//     allocate and synchronise the device. Make one warm-up call per device outside the step
//     loop, before any stream capture; later calls only launch and copy.
//   * Fields are real: a complex (Bloch) plan's imaginary parts are not read, so those
//     callers must use oem_plan_energy.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "oem_internal.cuh"

namespace {

constexpr int kMaxBlocks = oem::kEnergyMaxBlocks;  // block partial sums per call
constexpr int kMaxAxisCells = 32768;   // nx + ny + nz
constexpr int kPartials = 0;                       // [3 * kMaxBlocks] block partials
constexpr int kTotals = 3 * kMaxBlocks;            // [3] final sums
constexpr int kSpacing = kTotals + 3;              // [2 * kMaxAxisCells] primal / dual spacings
constexpr int kScratchDoubles = kSpacing + 2 * kMaxAxisCells;

static __device__ __align__(256) double g_energy_scratch[kScratchDoubles];

std::mutex g_setup_mu;
double* g_scratch_ptr[64] = {nullptr};

struct FieldSet {
  const float* f[6];
  const float* eps[3];  // nullptr = relative permittivity 1
};

// The per-block partial sums of oem_plan_energy's kernel (oem_kernels.cu), with the
// permittivity read from per-cell arrays instead of the material table.
__global__ void __launch_bounds__(256) k_energy_static(FieldSet F, int nx, int ny, int nz, int nzp,
                                                       double* scratch) {
  __shared__ double sh[3][256];
  const double* dxp = scratch + kSpacing;
  const double* dxd = dxp + nx;
  const double* dyp = dxd + nx;
  const double* dyd = dyp + ny;
  const double* dzp = dyd + ny;
  const double* dzd = dzp + nz;
  const int64_t n = (int64_t)nx * ny * nz;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % nz);
    const int64_t r = t / nz;
    const int j = (int)(r % ny);
    const int i = (int)(r / ny);
    const int64_t id = ((int64_t)i * ny + j) * nzp + k;
    const double vex = dxp[i] * dyd[j] * dzd[k];
    const double vey = dxd[i] * dyp[j] * dzd[k];
    const double vez = dxd[i] * dyd[j] * dzp[k];
    const double ex = F.f[0][id], ey = F.f[1][id], ez = F.f[2][id];
    const double hx = F.f[3][id], hy = F.f[4][id], hz = F.f[5][id];
    const double e0 = vex * ex * ex, e1 = vey * ey * ey, e2 = vez * ez * ez;
    const float p0 = F.eps[0] ? F.eps[0][id] : 1.0f;
    const float p1 = F.eps[1] ? F.eps[1][id] : 1.0f;
    const float p2 = F.eps[2] ? F.eps[2][id] : 1.0f;
    s0 += e0 + e1 + e2;
    s1 += e0 * p0 + e1 * p1 + e2 * p2;
    s2 += vex * hx * hx + vey * hy * hy + vez * hz * hz;  // H weighted like E
  }
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  sh[2][threadIdx.x] = s2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
      sh[2][threadIdx.x] += sh[2][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    scratch[kPartials + 3 * blockIdx.x + 0] = sh[0][0];
    scratch[kPartials + 3 * blockIdx.x + 1] = sh[1][0];
    scratch[kPartials + 3 * blockIdx.x + 2] = sh[2][0];
  }
}

// Sum the block partials in block order (the order oem_plan_energy sums them on the host).
__global__ void k_energy_total(int nblocks, double* scratch) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double a = 0.0, b = 0.0, c = 0.0;
  for (int q = 0; q < nblocks; ++q) {
    a += scratch[kPartials + 3 * q + 0];
    b += scratch[kPartials + 3 * q + 1];
    c += scratch[kPartials + 3 * q + 2];
  }
  scratch[kTotals + 0] = a;
  scratch[kTotals + 1] = b;
  scratch[kTotals + 2] = c;
}

// Device address of the scratch array for the current device, looked up once per device.
int scratch_for_current_device(double** out) {
  int dev = 0;
  OEM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return oem::set_error(OEM_ERR_INVALID, "device index above 63");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_energy_scratch);
    if (e != cudaSuccess) return oem::cuda_error(e, "cudaGetSymbolAddress(g_energy_scratch)");
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return OEM_OK;
}

}  // namespace

extern "C" int oem_field_energy_noalloc(const float* const fields[6], const float* const eps[3],
                                        int nx, int ny, int nz, int nzp, const double* spacing,
                                        double out[3], void* stream) {
  using oem::set_error;
  if (!fields || !spacing || !out) return set_error(OEM_ERR_INVALID, "null argument");
  for (int c = 0; c < 6; ++c)
    if (!fields[c]) return set_error(OEM_ERR_INVALID, "null field pointer");
  if (nx < 1 || ny < 1 || nz < 1 || nzp < nz)
    return set_error(OEM_ERR_INVALID, "bad grid dimensions (need nx, ny, nz >= 1, nzp >= nz)");
  if ((int64_t)nx + ny + nz > kMaxAxisCells)
    return set_error(OEM_ERR_INVALID,
                     "nx + ny + nz = " + std::to_string((int64_t)nx + ny + nz) +
                         " exceeds the no-allocation limit of " +
                         std::to_string(kMaxAxisCells) + " spacing entries");
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t nsp = 2 * ((size_t)nx + ny + nz);
  OEM_CUDA(cudaMemcpyAsync(scratch + kSpacing, spacing, nsp * sizeof(double),
                           cudaMemcpyHostToDevice, s));
  FieldSet F;
  for (int c = 0; c < 6; ++c) F.f[c] = fields[c];
  for (int c = 0; c < 3; ++c) F.eps[c] = eps ? eps[c] : nullptr;
  const int64_t n = (int64_t)nx * ny * nz;
  int64_t nb = (n + 255) / 256;
  if (nb > kMaxBlocks) nb = kMaxBlocks;
  if (nb < 1) nb = 1;
  k_energy_static<<<(unsigned)nb, 256, 0, s>>>(F, nx, ny, nz, nzp, scratch);
  OEM_CUDA(cudaGetLastError());
  k_energy_total<<<1, 1, 0, s>>>((int)nb, scratch);
  OEM_CUDA(cudaGetLastError());
  OEM_CUDA(cudaMemcpyAsync(out, scratch + kTotals, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return OEM_OK;
}
