// tild_internal.cuh — device state of a TILD engine (one or many independent systems on one
// GPU) and the device helpers shared by the kernels of libtild.
//
// An engine holds S systems that share dim and pmeorder.  Every per-step kernel covers all
// systems in one launch: particle kernels map a CTA (256 slots) to one system through a lookup
// table, grid kernels map a CTA of grid points the same way, and the FFTs run as one batched
// cuFFT plan per grid shape ("bucket").  A single-system context is an engine with S = 1.
//
// HBM layout (all arrays concatenated over systems; per-system offsets live in SysDev):
//   pos[2]     float4[NSP]  (x, y, z, type bits in .w); pos[cur] = x_n, pos[cur^1] = x_{n-1}
//              NSP = sum over systems of ns rounded up to 256; padding slots carry type 0xff
//   noise      float[3*NSP] GJF previous noise (reference d_prev_noise)
//   bead_id    int[NSP]     bead index within its system (-1 for padding)
//   bond_nbr   int[3*NSP]   partner slots (absolute); bond_info int[NSP] = n | t0<<8 | t1<<16 | t2<<24
//   rho_fx     u64[CH*M]    fixed-point density accumulators, CH channels = T + C per system
//   rho        f32[CH*M]    densities (x fastest like the reference)
//   rhok       c64[CH*Mh]   R2C of rho
//   gk         c64[CH*D*Mh] -i k_d Phi_t(k): input of the batched C2R
//   gfield     f32[CH*D*M]  -grad of the convolved potential (and E field), planar
//   g4         float4[CH*M] the same interleaved per grid point for the gather
//   utab       f32[sum nfft*Mh]          u_s(k)/M per FFT pair style
//   virk       c64[sum nfft*nP*Mh]       virial kernels / M^2
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <curand_kernel.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <atomic>
#include "../../include/tild.h"

#define TILD_MAXT_FAST 4   // k-space kernels are specialised for up to this many channels

// Device status word bits (reference: die() / NaN checks; here a flag the host polls).
enum : int {
  ST_NONFINITE_POS = 1,
  ST_INDEX_RANGE = 2,
  ST_NLIST_OVERFLOW = 4,
};

constexpr int kTile = 256;            // slots per particle CTA (systems are padded to it)
constexpr int kPadType = 0xff;        // type bits of a padding slot

struct Geom {
  int nx[3];
  int nxh;          // Nx/2 + 1
  float dx[3];      // L / Nx in FP32 (initialize.cu:36)
  float L[3];
  float Lh[3];      // 0.5f * L (config_utils.cu:46)
  float gvol;       // product of dx
  long long M, Mh;
};

// Per-system descriptor read by the kernels (one per system, in device memory).
struct SysDev {
  Geom g;
  int T, C, kbits, nfft;
  int slot0, ns, ns_pad, bead0;
  int slot_rank;                   // position of the system's slot range (the sort keeps the ranges)
  int active;                      // 0: skipped by the particle kernels
  long long grid0;                 // channel 0 of this system in rho / rho_fx / g4 (grid points)
  long long spec0;                 // channel 0 in rhok (half-spectrum points)
  int inv_packed;                  // 1: inverse transforms pair channels (2c, 2c+1) into one complex C2C
  long long gkp0;                  // with inv_packed: this system's first pair spectrum in gk (complex elements)
  int fwd_packed;                  // 1: densities of channels (2c, 2c+1) are stored as one complex field
                                   //    (real, imaginary) and take one forward C2C
  long long rkp0;                  // with fwd_packed: this system's first pair spectrum in rhok (complex elements)
  long long g4_0, Mb;              // channel 0 in g4 and the per-channel stride there (>= M)
  long long utab0, ctab0, kd0;     // offsets in utab, ctab, kd
  long long step;                  // completed steps (advanced on the device)
  long long stop_at;               // the system turns inactive once step reaches it (-1: never)
  int max_steps;
  int sa[TILD_MAX_STYLES], sb[TILD_MAX_STYLES], sramp[TILD_MAX_STYLES];
  float sAi[TILD_MAX_STYLES], sAf[TILD_MAX_STYLES], suk0[TILD_MAX_STYLES];
  uint64_t seed;
  float delt, noise_mag;
  int n_integ;
  int integ_kind[TILD_MAX_INTEGRATORS];
  int type_mask[TILD_MAX_TYPES];
  float mass[TILD_MAX_TYPES], diff[TILD_MAX_TYPES];
  float bond_k[TILD_MAX_BOND_TYPES], bond_req[TILD_MAX_BOND_TYPES];
};

struct FieldK {     // one fieldphase style
  int sys, a, b;
  int cfg_index;
  long long fr0;    // offset of its static field in frfield
};

// Host-side bookkeeping of one system.
struct SysHost {
  tild_config cfg;
  int D = 3, T = 1, C = 0, ns = 0, p = 1, S = 1, nP = 6;
  Geom g;
  double dV = 1.0, V = 1.0;
  int slot0 = 0, ns_pad = 0, bead0 = 0;  // bead0: first bead in the engine's bead numbering
  int cap = 0;                           // beads the slot can hold (>= ns; tild_batch_load)
  long long grid0 = 0, spec0 = 0, utab0 = 0, ctab0 = 0, kd0 = 0, virk0 = 0;
  long long g4_0 = 0, Mb = 0;            // force-field storage (tild_field_stride)
  int kbits = 20;
  std::vector<int> fft_cfg;              // fft table slot -> config style index
  int type_integ_mask[TILD_MAX_TYPES] = {0};
  int bucket = 0;
  int64_t step = 0, forces_step = 0;
  bool topo_set = false, state_set = false, have_forces = false, active = true;
  double* sk[TILD_MAX_COMPUTES] = {nullptr};
  int sk_calls[TILD_MAX_COMPUTES] = {0};
};

struct Bucket {     // systems sharing one grid shape: one batched R2C plan and one batched inverse
  int nx[3];
  std::vector<int> systems;
  long long grid0 = 0, spec0 = 0;        // first channel of the bucket
  int channels = 0;
  // inverse: C2R per channel and direction, or (packed) one complex C2C per channel pair and
  // direction whose real and imaginary parts are the pair's two real force fields
  bool packed = false;
  bool fwd_packed = false;               // the forward transforms pair channels too (out of place C2C)
  cufftHandle r2c = 0, c2r = 0, c2c = 0, c2c_fwd = 0;
  bool planned = false;
  int cta_spec0 = 0, n_cta_spec = 0;     // the shape's range of spectrum blocks (k-space multiply)
  int cta_grid0 = 0, n_cta_grid = 0;     // and of grid blocks (interleave)
  int cta_bead0 = 0, n_cta_bead = 0;     // and of particle blocks (spread, gather)
  int lane = 0;                          // auxiliary stream index (-1: main stream)
};

struct tild_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // auxiliary streams: the FFTs of different grid shapes run concurrently (fork/join by events)
  std::vector<cudaStream_t> aux;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  int lanes = 0;                         // auxiliary streams in use (tild_assign_lanes)
  // tunables (tild_autotune): spread kernel for order >= 2 and its shared box, in 32-bit words
  int spread_mode = TILD_SPREAD_TILED;
  int gather_mode = TILD_GATHER_DIRECT;  // order >= 2: stencil reads from global memory or shared boxes
  int gather_cap = 2048;                 // float4 nodes of a gather box buffer, 1024..3072
  int sort_brick = 0;                    // brick shape and order of the sort keys (tild_sort.cu)
  int field_layout = TILD_FIELD_LINEAR;  // node order of the float4 force field g4
  int fft_pipeline = 0;                  // per shape on its stream: 1 the grid stages, 2 the whole step
  int spread_ahead = 1;                  // integrating gathers spread x_{n+1} for the next step (order <= 1 default)
  bool rho_ahead = false;                // rho_fx already holds the densities of the current positions
  long long g4_total = 0;
  int D = 3, P = 1;
  int nsys = 1;
  std::vector<SysHost> sys;
  std::vector<Bucket> buckets;
  std::vector<FieldK> fields;
  SysDev* d_sys = nullptr;
  std::vector<SysDev> h_sys;             // host mirror of d_sys
  int rng = TILD_RNG_PHILOX;
  int maxT = 1;                          // largest channel count of a system (T + C)
  bool any_charges = false;

  // lookup tables: CTA -> system
  int* cta_bead = nullptr;  int n_cta_bead = 0;    // 256-slot blocks
  int* cta_spec = nullptr;  int n_cta_spec = 0;    // 256-point blocks of half spectra
  int* cta_grid = nullptr;  int n_cta_grid = 0;    // 256-point blocks of real grids
  std::vector<long long> spec_block0, grid_block0; // first block of each system

  // bead state
  int nslots = 0;
  float4* pos[2] = {nullptr, nullptr};
  int cur = 0;
  float* noise = nullptr;
  int* bead_id = nullptr;
  int* slot_of = nullptr;                // engine bead index -> slot
  int* bond_nbr = nullptr;
  int* bond_info = nullptr;
  float* charge = nullptr;
  int* types_dev = nullptr;
  curandStateXORWOW_t* xorwow = nullptr;
  int nbeads = 0;

  // grids
  long long grid_total = 0, spec_total = 0;  // channels x points
  unsigned long long* rho_fx = nullptr;
  float* rho = nullptr;
  cufftComplex* rhok = nullptr;
  cufftComplex* gk = nullptr;
  float* gfield = nullptr;
  float4* g4 = nullptr;
  float* utab = nullptr;
  float* ctab = nullptr;
  cufftComplex* virk = nullptr;
  float* frfield = nullptr;
  float* kd = nullptr;                   // derivative k per axis per system, Nyquist = 0
  float* kk = nullptr;                   // k per axis per system

  // scratch
  double* red = nullptr;
  int red_cap = 0;
  float* xfer = nullptr;                 // staging for host transfers, >= 3 * max ns floats
  int* d_status = nullptr;

  // spatial sort (tild_sort.cu)
  unsigned* sort_keys = nullptr;
  unsigned* sort_keys_alt = nullptr;
  int* sort_vals = nullptr;
  int* sort_perm = nullptr;
  int* sort_newslot = nullptr;
  int* slot_sys = nullptr;               // system of each slot
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
  int sort_cell_bits = 0;
  int sort_interval = 0;                 // 0: never
  int64_t steps_since_sort = 0;
  long long sorts = 0;
  int spread_cap = 0;                    // shared-memory 32-bit words of the tiled spread

  // CUDA graphs of whole step periods (tild_api.cu): keyed by the buffer configuration
  struct GraphEntry {
    cudaGraphExec_t exec;
    const void* p0;
    int cur;
    std::vector<char> buckets_on;        // grid shapes whose transforms the graph runs
    bool ahead, ahead_end;               // rho_ahead before and after the graph's steps
    int len;                             // steps in the graph
    int64_t sss0, sss_end;               // steps_since_sort before and after
    int cur_end;                         // buffer rotation after
    int nsorts;                          // sorts inside (each trades every per-slot array once)
    long long launches;                  // libtild kernel launches inside
  };
  std::vector<GraphEntry> graphs;
  bool use_graphs = true;
  int graph_len = 32;                    // graph length when the sort is disabled
  long long graph_launches_per_step = 0;

  // per-stage timing (tild_profile_steps)
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_stage;
  bool profiling = false;

  // FP64 table builds (tild_tables.cu): scratch sized for the largest grid, plans per grid shape
  struct TablePlan {
    int nx[3];
    cufftHandle z2d, d2z;
  };
  std::vector<TablePlan> tab_plans;
  long long tab_M = 0;
  double* tab_ufull = nullptr;
  cufftDoubleComplex* tab_z = nullptr;
  cufftDoubleComplex* tab_z2 = nullptr;
  double* tab_freal = nullptr;
  double* tab_vr = nullptr;

  bool any_stop = false;                 // some system has a device-side stop step

  // asynchronous snapshots (tild_snapshot_async): device buffers captured in stream order, copied
  // to the host on snap_stream; slot = ticket % TILD_SNAPSHOT_SLOTS
  struct SnapSlot {
    float* dx = nullptr;
    float* drho = nullptr;
    cudaEvent_t captured = nullptr, done = nullptr;
    std::atomic<long long> ticket{-1};
  };
  cudaStream_t snap_stream = nullptr;
  SnapSlot snaps[TILD_SNAPSHOT_SLOTS];
  long long snap_next = 0;
  size_t snap_x_floats = 0, snap_rho_floats = 0;

  long long launches = 0;
  std::string err;
};

enum TildStage {
  STAGE_SORT = 0, STAGE_ZERO, STAGE_SPREAD, STAGE_R2C, STAGE_KMUL, STAGE_C2R, STAGE_FIELD, STAGE_INTERLEAVE, STAGE_GATHER,
  STAGE_TAIL, STAGE_COUNT
};
static const char* const kStageNames[STAGE_COUNT] = {"sort", "fix2float", "spread", "r2c", "kmul", "c2r", "fieldphase", "interleave", "gather", "step_tail"};

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
// Per-channel storage of the float4 force field: room for the brick layout (3D: 4x4x4 bricks,
// edges rounded up to 4), so either layout fits without reallocating.
inline long long tild_field_stride(const Geom& g, int D) {
  if (D != 3) return g.M;
  return (long long)((g.nx[0] + 3) / 4) * ((g.nx[1] + 3) / 4) * ((g.nx[2] + 3) / 4) * 64;
}

// Offset of node n along axis d in one channel of the force field.  Linear: x fastest.  Brick
// (3D): 4x4x4 bricks of 64 consecutive nodes (1 KB), bricks x fastest, so the stencil loads of a
// warp of spatially sorted beads fall in a few contiguous blocks.
__device__ __forceinline__ int tild_field_off(int layout, int d, int n, const Geom& g) {
  if (layout == TILD_FIELD_LINEAR) return d == 0 ? n : (d == 1 ? n * g.nx[0] : n * g.nx[0] * g.nx[1]);
  const int nbx = (g.nx[0] + 3) >> 2, nby = (g.nx[1] + 3) >> 2;
  if (d == 0) return ((n >> 2) << 6) | (n & 3);
  if (d == 1) return (((n >> 2) * nbx) << 6) | ((n & 3) << 2);
  return (((n >> 2) * nbx * nby) << 6) | ((n & 3) << 4);
}
__device__ __forceinline__ int tild_type_of(float w) { return __float_as_int(w) & 0xff; }

// One channel of a paired density spectrum: Z = X_a + i X_b with X_a, X_b the spectra of two real
// fields, z = Z(k), zm = Z(-k); X_a(k) = (z + conj zm) / 2 (second = 0), X_b(k) = (z - conj zm) / 2i.
__device__ __forceinline__ float2 pair_unpack(float2 z, float2 zm, int second) {
  return second ? make_float2(0.5f * (z.y + zm.y), 0.5f * (zm.x - z.x))
                : make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
}

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

// Grid index of one bead along one axis (device_grid_utils.cu:256-266): even orders use the
// nearest node, odd orders the containing cell; returns the first stencil node and sets gdx, the
// offset from that node or cell centre that the spline weights take.
template <int P>
__device__ __forceinline__ int axis_index(float xj, float dxj, float& gdx) {
  int gi;
  if (P % 2 == 0) {
    gi = (int)((xj + 0.5f * dxj) / dxj);
    gdx = xj - (float)gi * dxj;
  } else {
    gi = (int)(xj / dxj);
    gdx = xj - ((float)gi + 0.5f) * dxj;
  }
  return gi - P / 2;
}

// Grid index and weights of one bead along one axis.
template <int P>
__device__ __forceinline__ int axis_base(float xj, float dxj, float* W) {
  float gdx;
  const int b = axis_index<P>(xj, dxj, gdx);
  spline_w<P>(gdx, dxj, W);
  return b;
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

// Ramp multiplier of FFT style k of a system for a force evaluation at `step`
// (PairStyle::Update, pair_style.cu:347-367: after every update u_k(0) equals
// A_i + (A_i - A_f) * (step + 1) / max_steps; forces of step n >= 2 see the update of n - 1).
__host__ __device__ inline float ramp_ratio(const SysDev& d, int k, long long step) {
  if (!d.sramp[k] || step < 2 || d.max_steps <= 0) return 1.0f;
  const double Ai = d.sAi[k], Af = d.sAf[k];
  const double target = Ai + (Ai - Af) * (double)step / (double)d.max_steps;
  return (float)(target / (double)d.suk0[k]);
}

// ---- host-side entry points between translation units ------------------------------------
int tild_build_tables(tild_ctx* c, int s);            // tild_tables.cu
int tild_run_forces(tild_ctx* c, bool integrate, float* f_bead, int f_sys);   // tild_step.cu
int tild_finish_forces(tild_ctx* c, bool integrate, float* f_bead, int f_sys, bool interleaved, bool gathered);
int tild_density_planar(tild_ctx* c, int s, float* dst, cudaStream_t st);                 // tild_step.cu
const float2* tild_half_spectra(tild_ctx* c, int s);                                     // tild_step.cu
int tild_obs_compute(tild_ctx* c, int s, tild_obs* o); // tild_obs.cu
int tild_sk_acc_run(tild_ctx* c, int s, int slot, int type);
int tild_table_scratch(tild_ctx* c);
int tild_assign_lanes(tild_ctx* c, int lanes);
int tild_drop_ahead(tild_ctx* c);                     // positions changed on the host: clear rho_fx

// Grid shapes with at least one active system: integrating steps skip the transforms of the others
// (their systems neither move nor are gathered).  Force-only evaluations transform every shape.
inline std::vector<char> tild_buckets_on(const tild_ctx* c) {
  std::vector<char> on(c->buckets.size(), 0);
  for (size_t b = 0; b < c->buckets.size(); b++)
    for (int s : c->buckets[b].systems)
      if (c->sys[s].active) {
        on[b] = 1;
        break;
      }
  return on;
}

// Whether this force evaluation's gather also spreads the updated positions into rho_fx for the
// next step (integrating steps with the direct gather; the box gather keeps its shared memory
// for the field).
inline bool tild_spreads_ahead(const tild_ctx* c, bool integrate) {
  return integrate && c->spread_ahead &&
         !(c->P >= 2 && c->gather_mode == TILD_GATHER_BOX && c->field_layout == TILD_FIELD_LINEAR);
}

// Brick shapes of the spatial sort the tuner chooses from (log2 edges x | y<<4 | z<<8, bit 12 =
// Morton order of the bricks); the first is the default.
inline std::vector<int> tild_brick_candidates(int D) {
  if (D == 3) return {0x222, 0x1222, 0x1113, 0x1123};
  return {0x033, 0x1033, 0x1014};
}


int tild_table_plans(tild_ctx* c, const Geom& g, int D, cufftHandle* z2d, cufftHandle* d2z);
void tild_tables_free(tild_ctx* c);
int tild_stencil_run(tild_ctx* c, int s, int* inds_dev, float* w_dev);
int tild_nlist_geom(const SysHost& h, float rc, int* nc, float* Lc, int* total, int* cmax);
int tild_nlist_run(tild_ctx* c, int s, float rc, int group_type, int* cell_of_bead_dev, int* ncount_dev,
                   int* neigh_dev);
int tild_check(tild_ctx* c, cudaError_t e, const char* what);
int tild_check_fft(tild_ctx* c, cufftResult r, const char* what);
int tild_poll_status(tild_ctx* c);
int tild_ensure_red(tild_ctx* c, int nvals, int nblocks);
int tild_sort_alloc(tild_ctx* c);                     // tild_sort.cu
void tild_sort_free(tild_ctx* c);
int tild_sort_beads(tild_ctx* c);
void tild_sort_swap_buffers(tild_ctx* c);
int tild_upload_sys(tild_ctx* c);                     // tild_api.cu: copies h_sys to d_sys
