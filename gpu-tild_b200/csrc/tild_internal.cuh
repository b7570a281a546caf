// tild_internal.cuh — device state of one TILD system and the device helpers shared by the
// kernels of libtild.
//
// HBM layout of a context (ns beads, M = prod(Nx) grid points, Mh = M/Nx*(Nx/2+1) half-spectrum
// points, T types, C = 1 with charges, D = dim):
//   pos[2]     float4[ns]   (x, y, z, type bits in .w); pos[cur] = x_n, pos[cur^1] = x_{n-1}
//   noise      float[ns*3]  GJF previous noise (reference d_prev_noise)
//   bead_id    int[ns]      original bead index of each slot (slots are re-ordered by the sort)
//   bond_nbr   int[ns*3]    partner slots; bond_info int[ns] = n | t0<<8 | t1<<16 | t2<<24
//   rho        float[(T+C)*M]        densities (spread), x fastest like the reference
//   rhok       cufftComplex[(T+C)*Mh] R2C of rho
//   gk         cufftComplex[(T+C)*D*Mh] -i k_d Phi_t(k): input of the batched C2R
//   gfield     float[(T+C)*D*M]      -grad of the convolved potential per type (and E field)
//   g4         float4[(T+C)*M]       the same, interleaved per grid point for the gather
//   utab       float[nfft_styles*Mh]  u_s(k)/M per FFT pair style
//   virk       cufftComplex[nfft_styles*nP*Mh] virial kernels / M^2
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <curand_kernel.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "../../include/tild.h"

#define TILD_MAXT_FAST 4   // kernels are specialised for up to this many channels

// Device status word bits (reference: die() / NaN checks; here a flag the host polls).
enum : int {
  ST_NONFINITE_POS = 1,
  ST_INDEX_RANGE = 2,
  ST_NLIST_OVERFLOW = 4,
};

struct Geom {
  int nx[3];
  int nxh;          // Nx/2 + 1
  float dx[3];      // L / Nx in FP32 (initialize.cu:36)
  float L[3];
  float Lh[3];      // 0.5f * L (config_utils.cu:46)
  float gvol;       // product of dx
  long long M, Mh;
};

struct StyleK {     // one FFT pair style as the k-space kernels see it
  int a, b;         // types
  int ramp;
  float Ai, Af;     // prefactors for the ramp
  float uk0;        // u_k(0) of the unscaled table (ramp denominator)
};

struct FieldK {     // one fieldphase style
  int a, b;
  int slot;         // index into frfield
};

struct tild_ctx {
  tild_config cfg;
  int device = 0;
  cudaStream_t stream = nullptr;
  int D = 3, T = 1, C = 0, ns = 0, p = 1, S = 1, nP = 6;
  Geom g;
  double dV = 1.0, V = 1.0;
  int max_steps = 0;

  // style bookkeeping
  std::vector<int> fft_style_index;   // config style index -> fft table slot (-1 if fieldphase)
  std::vector<StyleK> styles_k;       // per fft table slot
  std::vector<int> fft_style_cfg;     // fft table slot -> config style index
  std::vector<FieldK> fields;
  int type_integ_mask[TILD_MAX_TYPES] = {0};

  // bead state
  float4* pos[2] = {nullptr, nullptr};
  int cur = 0;
  float* noise = nullptr;
  int* bead_id = nullptr;
  int* slot_of = nullptr;
  int* bond_nbr = nullptr;
  int* bond_info = nullptr;
  float* charge = nullptr;
  float* bondk_dev = nullptr;         // bond constants [TILD_MAX_BOND_TYPES]
  float* bondr_dev = nullptr;
  int* types_dev = nullptr;           // per bead (bead order), kept for re-packing
  curandStateXORWOW_t* xorwow = nullptr;

  // grids
  unsigned long long* rho_fx = nullptr;  // fixed-point (2^32) density accumulator [(T+C)*M]
  float* rho = nullptr;
  cufftComplex* rhok = nullptr;
  cufftComplex* gk = nullptr;
  float* gfield = nullptr;
  float4* g4 = nullptr;                  // interleaved force field [(T+C)][M] (gather input)
  float* utab = nullptr;
  float* ctab = nullptr;              // charge force multiplier [Mh]
  cufftComplex* virk = nullptr;
  float* frfield = nullptr;           // [nfields*D*M]
  float* kd = nullptr;                // derivative k per axis: [nx0 + nx1 + nx2], Nyquist = 0
  float* kk = nullptr;                // k per axis for k^2: [nx0 + nx1 + nx2]

  // scratch for reductions and host transfers
  double* red = nullptr;              // partial sums
  int red_cap = 0;
  double* sk[TILD_MAX_COMPUTES] = {nullptr};
  int sk_calls[TILD_MAX_COMPUTES] = {0};
  float* xfer = nullptr;              // ns*4 floats staging (bead order)
  int* d_status = nullptr;

  cufftHandle plan_r2c = 0, plan_c2r = 0;
  bool plans = false;

  // spatial sort of the slots (tild_sort.cu)
  unsigned* sort_keys = nullptr;
  unsigned* sort_keys_alt = nullptr;
  int* sort_vals = nullptr;
  int* sort_perm = nullptr;
  int* sort_newslot = nullptr;
  float4* alt_pos[2] = {nullptr, nullptr};
  float* alt_noise = nullptr;
  int* alt_bead_id = nullptr;
  int* alt_info = nullptr;
  int* alt_nbr = nullptr;
  float* alt_charge = nullptr;
  curandStateXORWOW_t* alt_xorwow = nullptr;
  void* sort_temp = nullptr;
  size_t sort_temp_bytes = 0;
  int sort_bits = 0;
  int sort_kg[7] = {0};
  int sort_interval = 0;               // 0: never
  int64_t last_sort_step = -1;
  long long sorts = 0;
  int spread_cap = 0;                  // shared-memory 32-bit words of the tiled spread
  int spread_kbits = 20;               // fractional bits of the shared 32-bit fixed point

  // per-stage timing (tild_profile_steps): an event is recorded at every stage boundary
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_stage;
  bool profiling = false;

  int64_t step = 0;
  int64_t forces_step = 0;
  bool topo_set = false, state_set = false, have_forces = false;
  long long launches = 0;
  std::string err;
};

enum TildStage { STAGE_SORT = 0, STAGE_ZERO, STAGE_SPREAD, STAGE_R2C, STAGE_KMUL, STAGE_C2R, STAGE_FIELD, STAGE_GATHER, STAGE_COUNT };
static const char* const kStageNames[STAGE_COUNT] = {"sort", "fix2float", "spread", "r2c", "kmul", "c2r", "fieldphase", "gather"};

// Records the start of a stage when profiling (the next mark, or the final one, ends it).
inline void tild_mark(tild_ctx* c, int stage) {
  if (!c->profiling) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, c->stream);
  c->prof_ev.push_back(e);
  c->prof_stage.push_back(stage);
}

// ---- small helpers -----------------------------------------------------------------------
__device__ __forceinline__ int tild_type_of(float w) { return __float_as_int(w) & 0xff; }

// spline_get_weights (device_grid_utils.cu:3-49), FP32, including the order-4 quirk
// sx3 = sx2*sx2 of line 39.
template <int P>
__device__ __forceinline__ void spline_w(float gdx, float H, float* W) {
  const float sx = gdx / H;
  if (P == 0) {
    W[0] = 1.f;
  } else if (P == 1) {
    W[0] = 0.5f - sx;
    W[1] = 0.5f + sx;
  } else if (P == 2) {
    const float sx2 = sx * sx;
    W[0] = 0.125f - 0.5f * sx + 0.5f * sx2;
    W[1] = 0.75f - sx2;
    W[2] = 0.125f + 0.5f * sx + 0.5f * sx2;
  } else if (P == 3) {
    const float sx2 = sx * sx, sx3 = sx2 * sx;
    W[0] = (1.f - 6.f * sx + 12.f * sx2 - 8.f * sx3) / 48.f;
    W[1] = (23.f - 30.f * sx - 12.f * sx2 + 24.f * sx3) / 48.f;
    W[2] = (23.f + 30.f * sx - 12.f * sx2 - 24.f * sx3) / 48.f;
    W[3] = (1.f + 6.f * sx + 12.f * sx2 + 8.f * sx3) / 48.f;
  } else {
    const float sx2 = sx * sx, sx3 = sx2 * sx2, sx4 = sx2 * sx2;
    W[0] = (1.f - 8.f * sx + 24.f * sx2 - 32.f * sx3 + 16.f * sx4) / 384.f;
    W[1] = (19.f - 44.f * sx + 24.f * sx2 + 16.f * sx3 - 16.f * sx4) / 96.f;
    W[2] = (115.f - 120.f * sx2 + 48.f * sx4) / 192.f;
    W[3] = (19.f + 44.f * sx + 24.f * sx2 - 16.f * sx3 - 16.f * sx4) / 96.f;
    W[4] = (1.f + 8.f * sx + 24.f * sx2 + 32.f * sx3 + 16.f * sx4) / 384.f;
  }
}

// Grid index and weights of one bead along one axis (device_grid_utils.cu:256-266): even
// orders use the nearest node, odd orders the containing cell; base = first stencil node.
template <int P>
__device__ __forceinline__ int axis_base(float xj, float dxj, float* W) {
  int gi;
  float gdx;
  if (P % 2 == 0) {
    gi = (int)((xj + 0.5f * dxj) / dxj);
    gdx = xj - (float)gi * dxj;
  } else {
    gi = (int)(xj / dxj);
    gdx = xj - ((float)gi + 0.5f) * dxj;
  }
  spline_w<P>(gdx, dxj, W);
  return gi - P / 2;
}

// Periodic index with the reference's single conditional wrap; anything still outside the
// grid (only possible for positions far outside [0,L]) is folded back and flagged.
__device__ __forceinline__ int wrap_idx(int n, int N, int* status) {
  if (n < 0) n += N;
  else if (n >= N) n -= N;
  if ((unsigned)n >= (unsigned)N) {
    atomicOr(status, ST_INDEX_RANGE);
    n %= N;
    if (n < 0) n += N;
  }
  return n;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11).  Counter = (step lo, step hi, integrator index, seed hi), key = (bead id, seed lo).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Three N(0,1) draws by Box-Muller from 24-bit uniforms (u0, u2 odd numerators: in (0,1)).
__device__ __forceinline__ void philox_normal3(uint64_t seed, uint32_t bead, int64_t step,
                                               uint32_t integ, float z[3]) {
  const uint4 r = philox4x32_10(
      make_uint4((uint32_t)step, (uint32_t)((uint64_t)step >> 32), integ, (uint32_t)(seed >> 32)),
      make_uint2(bead, (uint32_t)seed));
  const float u0 = (float)((r.x >> 8) | 1u) * 0x1p-24f;
  const float u1 = (float)(r.y >> 8) * 0x1p-24f;
  const float u2 = (float)((r.z >> 8) | 1u) * 0x1p-24f;
  const float u3 = (float)(r.w >> 8) * 0x1p-24f;
  const float r0 = sqrtf(-2.f * logf(u0)), r1 = sqrtf(-2.f * logf(u2));
  float s0, c0, s1, c1;
  sincospif(2.f * u1, &s0, &c0);
  sincospif(2.f * u3, &s1, &c1);
  z[0] = r0 * c0;
  z[1] = r0 * s0;
  z[2] = r1 * c1;
}

// ---- host-side entry points between translation units ------------------------------------
int tild_build_tables(tild_ctx* c);                   // tild_tables.cu
int tild_run_forces(tild_ctx* c, int64_t step, bool integrate, float* f_slot);  // tild_step.cu
int tild_run_spread(tild_ctx* c);                     // tild_step.cu
int tild_obs_compute(tild_ctx* c, tild_obs* o);       // tild_obs.cu
int tild_sk_acc_run(tild_ctx* c, int slot, int type);
int tild_stencil_run(tild_ctx* c, int* inds_dev, float* w_dev);
int tild_nlist_geom(const tild_ctx* c, float rc, int* nc, float* Lc, int* total, int* cmax);
int tild_nlist_run(tild_ctx* c, float rc, int group_type, int* cell_of_bead_dev, int* ncount_dev, int* neigh_dev);
int tild_check(tild_ctx* c, cudaError_t e, const char* what);
int tild_check_fft(tild_ctx* c, cufftResult r, const char* what);
int tild_poll_status(tild_ctx* c);
int tild_ensure_red(tild_ctx* c, int nvals, int nblocks);
int tild_sort_alloc(tild_ctx* c);                     // tild_sort.cu
void tild_sort_free(tild_ctx* c);
int tild_sort_beads(tild_ctx* c);
double tild_ramp_ratio(const tild_ctx* c, int fft_slot, int64_t step);
