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
//  * the array's device address is looked up (cudaGetSymbolAddress) on every call made outside
//    stream capture, so a device reset or a new primary context between calls is picked up;
//    a call made while its stream is capturing uses the address the last uncaptured call on
//    that device and context found, so make one call outside capture first (again after any
//    device reset);
//  * a CUDA error already pending on the calling thread is reported and left pending: the
//    call launches nothing and returns TILD_ERR_CUDA, and the caller's error is not consumed.
#include <cuda.h>
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
struct CachedAddr {
  double* addr = nullptr;
  void* ctx = nullptr;  // the context the address belongs to
};
CachedAddr g_partials[kMaxDevices];

// The calling thread's current context (driver entry point through the runtime, so the library
// needs no link against the driver library); nullptr when it cannot be had.
void* current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<Fn>(p);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

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
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    if (n < 0 || n > TILD_MAX_BONDS) v[0] = qnan;  // corrupt topology: poison the result
    for (int b = 0; b < n && b < TILD_MAX_BONDS; b++) {
      const int j = bto[3 * i + b];
      const int bt = bty[3 * i + b];
      if (j < 0 || j >= a.ns || bt < 0 || bt >= a.nbt) {  // checked before the j < i skip
        v[0] = qnan;
        continue;
      }
      if (j < i) continue;
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
  // an error left by earlier work on this thread is the caller's: report it, keep it pending
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    fprintf(stderr, "tild_bond_observables_noalloc: a CUDA error from earlier work is pending (%s); nothing launched\n",
            cudaGetErrorString(pending));
    return TILD_ERR_CUDA;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    fprintf(stderr, "tild_bond_observables_noalloc: no usable current device\n");
    return TILD_ERR_CUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    fprintf(stderr, "tild_bond_observables_noalloc: invalid stream\n");
    return TILD_ERR_BAD_INPUT;
  }
  void* ctx = current_context();
  double* partials = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mutex);
    CachedAddr& ca = g_partials[dev];
    if (cap == cudaStreamCaptureStatusNone) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_bond_partials);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        fprintf(stderr, "tild_bond_observables_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return TILD_ERR_CUDA;
      }
      ca.addr = static_cast<double*>(p);
      ca.ctx = ctx;
    } else if (!ca.addr || ca.ctx != ctx) {
      fprintf(stderr, "tild_bond_observables_noalloc: called under stream capture before any call outside capture "
                      "on this device and context\n");
      return TILD_ERR_STATE;
    }
    partials = ca.addr;
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
  k_bond_partials<<<nblocks, kThreads, 0, st>>>(d_x, d_n_bonds, d_bonded_to, d_bond_type, a, partials);
  k_bond_final<<<1, 32, 0, st>>>(partials, nblocks, 1.0 / V / (double)dim, np, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "tild_bond_observables_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return TILD_ERR_CUDA;
  }
  return TILD_OK;
}
