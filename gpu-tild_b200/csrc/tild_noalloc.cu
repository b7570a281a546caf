// tild_noalloc.cu — bond energy and virial for callers that cannot allocate device memory.
//
// Some callers of this library run where cudaMalloc is not theirs to call: code that executes
// inside another framework's memory pool or allocator-free plugin slot, hosts that forbid new
// device allocations after start-up, or a step that must not reach the allocator at all.
// They hold device arrays already (positions, topology) and only need a reduction over them.
// tild_bond_observables_noalloc gives them the bond energy and bond virial of host_bonds
// (bonds.cu:3-52) without allocating: its per-block partial sums live in the fixed array
// below, which every GPU that loads libtild holds for the life of the process.
//
// Limits and sharing:
//  * at most TILD_NOALLOC_MAX_BLOCKS blocks of 256 beads, i.e. TILD_NOALLOC_MAX_BEADS beads
//    per call; larger ns is rejected with TILD_ERR_BAD_INPUT before anything is launched;
//  * every call on a device uses the same array and leaves its partial sums there; each call
//    writes every slot it later reads, so no clearing is needed, but two calls whose kernels
//    overlap on the GPU (different streams, no ordering between them) race on the array;
//  * the first call on each device (with that device current) looks up the array's device
//    address; make that first call before any stream capture.
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>
#include "../../include/tild.h"

namespace {

constexpr int kThreads = 256;
constexpr int kVals = 7;  // energy + up to six virial components
constexpr int kMaxDevices = 64;

// The scratch: per-block partial sums.  In host code this name is only a stand-in for the
// device symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_bond_partials[TILD_NOALLOC_MAX_BLOCKS * kVals];

std::mutex g_mutex;
double* g_partials_addr[kMaxDevices] = {nullptr};

struct BondArgs {
  float L[3], Lh[3];
  float k[TILD_MAX_BOND_TYPES], req[TILD_MAX_BOND_TYPES];
  int nbt, ns, D;
};

// One thread per bead, every bond counted once (partner id >= own id, bonds.cu:141-143),
// FP64 accumulation, per-block partials written to `partials`.
__global__ void __launch_bounds__(kThreads) k_bond_partials(const float* __restrict__ x, const int* __restrict__ nb,
                                                           const int* __restrict__ bto, const int* __restrict__ bty,
                                                           BondArgs a, double* __restrict__ partials) {
  double v[kVals] = {0, 0, 0, 0, 0, 0, 0};
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ns) {
    const int n = nb[i];
    for (int b = 0; b < n && b < TILD_MAX_BONDS; b++) {
      const int j = bto[3 * i + b];
      const int bt = bty[3 * i + b];
      if (j < i) continue;
      if (j >= a.ns || bt < 0 || bt >= a.nbt) {  // corrupt topology: poison the result
        v[0] = __longlong_as_double(0x7ff8000000000000LL);
        continue;
      }
      double dr[3] = {0, 0, 0}, mdr2 = 0.0;
      for (int d = 0; d < a.D; d++) {
        const float xi = x[(long long)i * a.D + d], xj = x[(long long)j * a.D + d];
        const float drf = xi - xj;
        double dv = (double)xi - (double)xj;
        if (drf > a.Lh[d]) dv -= (double)a.L[d];
        else if (drf < -a.Lh[d]) dv += (double)a.L[d];
        dr[d] = dv;
        mdr2 += dv * dv;
      }
      const double mdr = sqrt(mdr2), delr = mdr - (double)a.req[bt];
      v[0] += delr * delr * (double)a.k[bt];
      const double mf = 2.0 * (double)a.k[bt] * delr / mdr;
      v[1] += -mf * dr[0] * dr[0];
      v[2] += -mf * dr[1] * dr[1];
      if (a.D == 2) {
        v[3] += -mf * dr[0] * dr[1];
      } else {
        v[3] += -mf * dr[2] * dr[2];
        v[4] += -mf * dr[0] * dr[1];
        v[5] += -mf * dr[0] * dr[2];
        v[6] += -mf * dr[1] * dr[2];
      }
    }
  }
  __shared__ double sh[kVals][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < kVals; k++) {
    double s = v[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh[k][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x < kVals) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; w++) s += sh[threadIdx.x][w];
    partials[(long long)blockIdx.x * kVals + threadIdx.x] = s;
  }
}

// Fixed-order sum of the partials (deterministic), scaled as host_bonds scales the virial.
__global__ void k_bond_final(const double* __restrict__ partials, int nblocks, double inv_vd, int np,
                             double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k > np) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; b++) s += partials[(long long)b * kVals + k];
  out[k] = (k == 0) ? s : s * inv_vd;
}

}  // namespace

extern "C" int32_t tild_bond_observables_noalloc(const float* d_x, const int32_t* d_n_bonds,
                                                 const int32_t* d_bonded_to, const int32_t* d_bond_type, int32_t ns,
                                                 int32_t dim, const float* box, int32_t n_bond_types,
                                                 const float* bond_k, const float* bond_req, double* d_out,
                                                 void* stream) {
  if (!d_x || !d_n_bonds || !d_bonded_to || !d_bond_type || !box || !bond_k || !bond_req || !d_out) {
    fprintf(stderr, "tild_bond_observables_noalloc: null argument\n");
    return TILD_ERR_BAD_INPUT;
  }
  if (dim != 2 && dim != 3) {
    fprintf(stderr, "tild_bond_observables_noalloc: dim must be 2 or 3\n");
    return TILD_ERR_BAD_INPUT;
  }
  if (n_bond_types < 1 || n_bond_types > TILD_MAX_BOND_TYPES) {
    fprintf(stderr, "tild_bond_observables_noalloc: n_bond_types must be 1..%d\n", TILD_MAX_BOND_TYPES);
    return TILD_ERR_BAD_INPUT;
  }
  if (ns < 0 || ns > TILD_NOALLOC_MAX_BEADS) {
    fprintf(stderr,
            "tild_bond_observables_noalloc: ns = %d exceeds the fixed scratch (at most %d beads per call)\n",
            (int)ns, (int)TILD_NOALLOC_MAX_BEADS);
    return TILD_ERR_BAD_INPUT;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    fprintf(stderr, "tild_bond_observables_noalloc: no usable current device\n");
    return TILD_ERR_CUDA;
  }
  double* partials = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mutex);
    if (!g_partials_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_bond_partials);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        fprintf(stderr, "tild_bond_observables_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return TILD_ERR_CUDA;
      }
      g_partials_addr[dev] = static_cast<double*>(p);
    }
    partials = g_partials_addr[dev];
  }
  BondArgs a;
  double V = 1.0;
  for (int d = 0; d < 3; d++) {
    a.L[d] = d < dim ? box[d] : 1.0f;
    a.Lh[d] = 0.5f * a.L[d];
    if (d < dim) V *= (double)a.L[d];
  }
  for (int b = 0; b < TILD_MAX_BOND_TYPES; b++) {
    a.k[b] = b < n_bond_types ? bond_k[b] : 0.f;
    a.req[b] = b < n_bond_types ? bond_req[b] : 0.f;
  }
  a.nbt = n_bond_types;
  a.ns = ns;
  a.D = dim;
  const int np = (dim == 2) ? 3 : 6;
  const int nblocks = ns > 0 ? (ns + kThreads - 1) / kThreads : 1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_bond_partials<<<nblocks, kThreads, 0, st>>>(d_x, d_n_bonds, d_bonded_to, d_bond_type, a, partials);
  k_bond_final<<<1, 32, 0, st>>>(partials, nblocks, 1.0 / V / (double)dim, np, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "tild_bond_observables_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return TILD_ERR_CUDA;
  }
  return TILD_OK;
}
