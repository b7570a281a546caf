// tild_step.cu — the per-step hot path over all systems of an engine: spread -> batched R2C ->
// k-space multiply -> batched C2R -> fused gather + bonds + integrators.
//
// Replaces forces() (forces.cu:42-196) followed by Integrator::Integrate_2()
// (integrator.cu:24-39).  Differences of formulation, each exact in real arithmetic:
//  * one R2C per density instead of two C2C per pair style and side, and one C2R per
//    (type, direction) instead of Dim C2C per style and side: the k-space kernel sums all
//    styles acting on a type first, Phi_I(k) = sum_J u_IJ(k) rho_J(k) / M (a self pair counts
//    twice, pair_style.cu:119-235 applies it to both sides);
//  * the gather reads -grad Phi_I directly instead of rho_I * (-grad Phi_I) / rho_I
//    (device_grid_utils.cu:424-452), fieldphase adds rho_I * f_r (its grid force rho_I^2 f_r
//    divided by rho_I, device_array_utils.cu:362-372 and 410-423);
//  * the derivative of the Nyquist plane is zero: the reference's Re() of a full C2C inverse
//    discards exactly those modes;
//  * stencil weights are recomputed in the gather rather than cached (no ns*S W/inds arrays).
// Each launch covers every system of the engine: CTAs find their system in a lookup table.
#include "tild_internal.cuh"
#include <climits>

namespace {

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

constexpr double kInvFix = 1.0 / 4294967296.0;  // the global accumulator holds 2^32 per unit
constexpr int kMaxRows = 1024;                  // (y, z) rows of a shared-memory spread box
constexpr int kGatherBoxMax = 3072;             // float4 nodes of the gather's shared box (48 KB)

// n mod N in [0, N); indices within one period of the grid (nearly all) take no division
__device__ __forceinline__ int pmod(int n, int N) {
  if ((unsigned)n < (unsigned)N) return n;
  if (n < 0 && n >= -N) return n + N;
  if (n >= N && n - N < N) return n - N;
  n %= N;
  return n < 0 ? n + N : n;
}

// r folded into (-N/2, N/2]
__device__ __forceinline__ int fold_rel(int r, int N) {
  r = pmod(r, N);
  if (r > N / 2) r -= N;
  return r;
}

// Chunk bounding box of the beads' stencil bases, relative to the chunk's first bead.
// Returns false when no bead of the chunk is valid.  Every thread of the block must call it.
template <int D, int P>
__device__ __forceinline__ bool chunk_box(bool ok, const int (&rel)[3], int* s_min, int* s_max, int (&mn)[3],
                                          int (&ext)[3], long long& vol) {
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int d = 0; d < D; d++) {
    const int a = __reduce_min_sync(full, ok ? rel[d] : INT_MAX);
    const int b = __reduce_max_sync(full, ok ? rel[d] : INT_MIN);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&s_min[d], a);
      atomicMax(&s_max[d], b);
    }
  }
  __syncthreads();
  if (s_max[0] < s_min[0]) return false;
  vol = 1;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    mn[d] = d < D ? s_min[d] : 0;
    ext[d] = d < D ? s_max[d] - s_min[d] + P + 1 : 1;
    vol *= ext[d];
  }
  return true;
}

template <int D, int P>
__device__ __forceinline__ void chunk_origin(const float4* __restrict__ pos, int i0, const Geom& g, int* s_g0,
                                             int* s_min, int* s_max) {
  if (threadIdx.x == 0) {
    const float4 p0 = pos[i0];
    const float x0[3] = {p0.x, p0.y, p0.z};
    const bool valid = tild_type_of(p0.w) != kPadType;
    float Wd[P + 1];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      s_g0[d] = (valid && d < D && isfinite(x0[d])) ? axis_base<P>(x0[d], g.dx[d], Wd) : 0;
      s_min[d] = INT_MAX;
      s_max[d] = INT_MIN;
    }
  }
  __syncthreads();
}

// One bead's stencil added to the 64-bit global accumulator (2^32 per unit) in contributions
// rounded at 2^kbits per unit, with the float operations of the shared-box path, so that a node's
// integer sum is the same whichever path (or spread kernel) a bead takes.
template <int D, int P>
__device__ __forceinline__ void spread_global_kbits(const float (&W)[3][P + 1], const int (&idx)[3][P + 1],
                                                    const Geom& g, unsigned long long* rt, unsigned long long* rc,
                                                    float q, float ig, int kbits) {
  const float sc32 = ig * __int_as_float((127 + kbits) << 23);  // 2^kbits / gvol
  const int sh = 32 - kbits;
#pragma unroll
  for (int ix = 0; ix <= P; ix++)
#pragma unroll
    for (int iy = 0; iy <= P; iy++) {
      const long long row = idx[0][ix] + (long long)idx[1][iy] * g.nx[0];
      const float wxy = W[0][ix] * W[1][iy] * sc32;
#pragma unroll
      for (int iz = 0; iz <= (D == 3 ? P : 0); iz++) {
        const long long m = D == 3 ? row + (long long)idx[2][iz] * g.nx[1] * g.nx[0] : row;
        const float W3 = D == 3 ? wxy * W[2][iz] : wxy;
        atomicAdd(rt + m, (unsigned long long)((long long)__float2int_rn(W3) << sh));
        if (rc) atomicAdd(rc + m, (unsigned long long)((long long)__float2int_rn(W3 * q) << sh));
      }
    }
}

// ---------------------------------------------------------------------------------------------
// Spreading: d_charge_grid / d_charge_grid_charges (device_grid_utils.cu:111-343)
// ---------------------------------------------------------------------------------------------
// One CTA takes 256 consecutive slots of one system; their stencil nodes are accumulated into a
// shared-memory box (relative to the first bead, periodic offsets folded into [-N/2, N/2]) and
// the box is added to the global grid once.  Accumulation is fixed point: the shared box holds
// 32-bit integers with 2^kbits per unit (native integer atomics; kbits is chosen per system so
// 256 beads at the largest weight cannot overflow), the global accumulator 64-bit integers with
// 2^32 per unit.  Integer sums do not depend on the order of the additions, so the densities are
// bitwise reproducible whatever the slot order or scheduling.  A chunk whose box does not fit
// adds each node to the global accumulator directly.
//
// The spread of one CTA's beads, positions already in registers (ok: this thread's bead is valid
// and finite; t its type; q its charge, 0 without).  Thread 0's bead is the box origin.  Every
// thread of the block must call it.  The spread kernel and the spreading gather share it.
template <int D, int P, bool CH>
__device__ __forceinline__ void cta_spread_box(bool ok, const float (&xs)[3], int t, float q, const SysDev& sd,
                                               unsigned long long* __restrict__ rho_fx, int cap, int* status) {
  extern __shared__ __align__(16) int smi[];  // the box: cap words, cap a multiple of 4
  __shared__ int s_g0[3], s_min[3], s_max[3];
  __shared__ int s_row[kMaxRows];  // row offsets in one channel (grids hold fewer than 2^31 points)
  const Geom g = sd.g;
  const int T = sd.T, C = sd.C, kbits = sd.kbits;
  if (threadIdx.x == 0) {
    float Wd[P + 1];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      s_g0[d] = (ok && d < D) ? axis_base<P>(xs[d], g.dx[d], Wd) : 0;
      s_min[d] = INT_MAX;
      s_max[d] = INT_MIN;
    }
  }
  __syncthreads();
  // only the per-axis spline offsets live across the box barriers; the weights come after them
  float gd[3] = {0.f, 0.f, 0.f};
  int rel[3] = {0, 0, 0};
  if (ok) {
#pragma unroll
    for (int d = 0; d < D; d++) rel[d] = fold_rel(axis_index<P>(xs[d], g.dx[d], gd[d]) - s_g0[d], g.nx[d]);
  }
  int mn[3], ext[3];
  long long vol;
  if (!chunk_box<D, P>(ok, rel, s_min, s_max, mn, ext, vol)) return;
  const int nch = T + C;
  const long long M = g.M;
  const float ig = 1.0f / g.gvol;
  const bool qc = CH && C && q != 0.f;
  if (vol * nch <= cap && ext[0] <= 64 && ext[1] * ext[2] <= kMaxRows) {
    const int tot = (int)vol * nch;
    {  // clear with 16-byte stores (the box buffer holds cap words, cap a multiple of 4)
      int4* s4 = reinterpret_cast<int4*>(smi);
      for (int k = threadIdx.x; k < (tot + 3) >> 2; k += blockDim.x) s4[k] = make_int4(0, 0, 0, 0);
    }
    __syncthreads();
    if (ok) {
      float W[3][P + 1];
#pragma unroll
      for (int d = 0; d < D; d++) spline_w<P>(gd[d], g.dx[d], W[d]);
      const float sc32 = ig * __int_as_float((127 + kbits) << 23);  // 2^kbits / gvol
      int* st = smi + (long long)t * vol;
      int* sq = smi + (long long)T * vol;
#pragma unroll
      for (int ix = 0; ix <= P; ix++)
#pragma unroll
        for (int iy = 0; iy <= P; iy++) {
          const int rowl = (rel[1] - mn[1] + iy) * ext[0] + (rel[0] - mn[0] + ix);
          const float wxy = W[0][ix] * W[1][iy] * sc32;
          if (D == 3) {
#pragma unroll
            for (int iz = 0; iz <= P; iz++) {
              const int l = (rel[2] - mn[2] + iz) * ext[1] * ext[0] + rowl;
              const float W3 = wxy * W[2][iz];
              atomicAdd(st + l, __float2int_rn(W3));
              if (qc) atomicAdd(sq + l, __float2int_rn(W3 * q));
            }
          } else {
            atomicAdd(st + rowl, __float2int_rn(wxy));
            if (qc) atomicAdd(sq + rowl, __float2int_rn(wxy * q));
          }
        }
    }
    __syncthreads();
    // row offsets of the box in one channel of the periodic grid
    const int rows_per = ext[1] * ext[2];
    for (int yz = threadIdx.x; yz < rows_per; yz += blockDim.x) {
      const int ly = yz % ext[1], lz = yz / ext[1];
      s_row[yz] = g.nx[0] * (pmod(s_g0[1] + mn[1] + ly, g.nx[1]) +
                             g.nx[1] * (D == 3 ? pmod(s_g0[2] + mn[2] + lz, g.nx[2]) : 0));
    }
    __syncthreads();
    // flush: every thread takes box words tid, tid + 256, ... of each channel (all lanes busy);
    // a word's row is k / ext0 by a multiply-high (exact: k < 2^26, ext0 >= 3), and each nonzero
    // word is shifted exactly onto the 2^32 grid and added with one 64-bit RED
    const int ex = ext[0];
    const unsigned mul = 0xFFFFFFFFu / (unsigned)ex + 1u;  // ceil(2^32 / ex)
    const int bx = pmod(s_g0[0] + mn[0], g.nx[0]);
    const int sh = 32 - kbits;
    for (int ch = 0; ch < nch; ch++) {
      const int* sch = smi + (long long)ch * vol;
      unsigned long long* gch = rho_fx + ch * M;
      for (int k = threadIdx.x; k < (int)vol; k += blockDim.x) {
        const int v = sch[k];
        if (v == 0) continue;
        const int row = (int)__umulhi((unsigned)k, mul);
        int xg = bx + (k - row * ex);
        while (xg >= g.nx[0]) xg -= g.nx[0];
        atomicAdd(gch + s_row[row] + xg, (unsigned long long)((long long)v << sh));
      }
    }
  } else if (ok) {
    // the box does not fit: the same 2^kbits contributions, added to the global grid directly
    float W[3][P + 1];
#pragma unroll
    for (int d = 0; d < D; d++) spline_w<P>(gd[d], g.dx[d], W[d]);
    int idx[3][P + 1];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int a = 0; a <= P; a++) idx[d][a] = pmod(s_g0[d] + rel[d] + a, g.nx[d]);
    spread_global_kbits<D, P>(W, idx, g, rho_fx + (long long)t * M, qc ? rho_fx + (long long)T * M : nullptr, q,
                              ig, kbits);
  }
}

// One valid, finite bead straight into the 64-bit global accumulator.  For order <= 1 (8-node
// stencils) the contributions keep 2^32 per unit; for higher orders they are rounded exactly as
// the box rounds them.
template <int D, int P, bool CH>
__device__ __forceinline__ void bead_spread_direct(const float (&xs)[3], int t, float q, const SysDev& sd,
                                                   unsigned long long* __restrict__ rho_fx_all) {
  const Geom& g = sd.g;
  const int T = sd.T;
  const long long M = g.M;
  float W[3][P + 1];
  int idx[3][P + 1];
#pragma unroll
  for (int d = 0; d < D; d++) {
    const int b = axis_base<P>(xs[d], g.dx[d], W[d]);
#pragma unroll
    for (int a = 0; a <= P; a++) idx[d][a] = pmod(b + a, g.nx[d]);
  }
  unsigned long long* rt = rho_fx_all + sd.grid0 + (long long)t * M;
  unsigned long long* rc = rho_fx_all + sd.grid0 + (long long)T * M;
  if (P >= 2) {  // same contributions as the shared-box path: results independent of the choice
    spread_global_kbits<D, P>(W, idx, g, rt, (CH && q != 0.f) ? rc : nullptr, q, 1.0f / g.gvol, sd.kbits);
    return;
  }
  const double sc64 = 4294967296.0 / (double)g.gvol;
#pragma unroll
  for (int ix = 0; ix <= P; ix++)
#pragma unroll
    for (int iy = 0; iy <= P; iy++) {
      const long long row = idx[0][ix] + (long long)idx[1][iy] * g.nx[0];
      const float wxy = W[0][ix] * W[1][iy];
#pragma unroll
      for (int iz = 0; iz <= (D == 3 ? P : 0); iz++) {
        const long long m = D == 3 ? row + (long long)idx[2][iz] * g.nx[1] * g.nx[0] : row;
        const double W3 = (double)(D == 3 ? wxy * W[2][iz] : wxy) * sc64;
        atomicAdd(rt + m, (unsigned long long)__double2ll_rn(W3));
        if (CH && q != 0.f) atomicAdd(rc + m, (unsigned long long)__double2ll_rn(W3 * q));
      }
    }
}

// a slot's bead for the spread: valid (not padding) and finite; a non-finite one is reported
template <int D, bool CH>
__device__ __forceinline__ bool spread_input(const float4& p, const SysDev& sd, const float* __restrict__ charge,
                                             int i, float (&xs)[3], int& t, float& q, int* status) {
  xs[0] = p.x;
  xs[1] = p.y;
  xs[2] = p.z;
  t = tild_type_of(p.w);
  q = 0.f;
  if (t == kPadType) return false;
  if (!(isfinite(p.x) && isfinite(p.y) && (D == 2 || isfinite(p.z)))) {
    atomicOr(status, ST_NONFINITE_POS);
    return false;
  }
  if (CH && sd.C) q = charge[i];
  return true;
}

// 7 CTAs per SM (32 registers, a few spilled): the barriers of one CTA's box phases are covered
// by the others (blend: 0.153 -> 0.144 ms against 48 registers and 5 CTAs)
template <int D, int P, bool CH>
__global__ void __launch_bounds__(256, 7) k_spread_tiled(const float4* __restrict__ pos, const float* __restrict__ charge,
                                                     const int* __restrict__ cta_sys,
                                                     const SysDev* __restrict__ sysd,
                                                     unsigned long long* __restrict__ rho_fx_all, int cap,
                                                     int* status, int blk_off) {
  const int blk = blockIdx.x + blk_off;
  const SysDev& sd = sysd[cta_sys[blk]];  // inactive systems too (see k_fix_to_float)
  static_assert(kTile == 256, "the lane-to-slot map below assumes 8 warps of 32");
  // lane l of warp w takes slot 8 l + w: a warp's beads lie in distinct cells, so its shared
  // atomics meet fewer equal addresses; thread 0 keeps slot 0, the box origin
  const int i = blk * blockDim.x + (((threadIdx.x & 31) << 3) | (threadIdx.x >> 5));
  float xs[3], q;
  int t;
  const bool ok = spread_input<D, CH>(pos[i], sd, charge, i, xs, t, q, status);
  cta_spread_box<D, P, CH>(ok, xs, t, q, sd, rho_fx_all + sd.grid0, cap, status);
}

// Every node straight into the 64-bit global accumulator: always for order <= 1, where a shared
// box would cost more to zero, synchronise and flush than its shared atomics save; for higher
// orders it is the tuner's alternative to the box.
template <int D, int P, bool CH>
__global__ void __launch_bounds__(256) k_spread_direct(const float4* __restrict__ pos, const float* __restrict__ charge,
                                                      const int* __restrict__ cta_sys, const SysDev* __restrict__ sysd,
                                                      unsigned long long* __restrict__ rho_fx_all, int* status,
                                                      int blk_off) {
  const int blk = blockIdx.x + blk_off;
  const SysDev& sd = sysd[cta_sys[blk]];  // inactive systems too (see k_fix_to_float)
  const int i = blk * blockDim.x + threadIdx.x;
  float xs[3], q;
  int t;
  if (spread_input<D, CH>(pos[i], sd, charge, i, xs, t, q, status))
    bead_spread_direct<D, P, CH>(xs, t, q, sd, rho_fx_all);
}

// fixed-point grid -> FP32 density over every system's channels, clearing the accumulator for the
// next step.  Inactive systems are spread too (their positions are held), so their densities stay
// those of their last step and their observables can still be read.
__global__ void k_fix_to_float(unsigned long long* __restrict__ fx, float* __restrict__ rho, long long n) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const long long v = (long long)fx[k];
  rho[k] = (float)((double)v * kInvFix);
  fx[k] = 0ull;
}

// The same conversion for a grid shape whose channels are paired: channels 2p and 2p + 1 of node m
// become the complex value (rho_2p, rho_2p+1) at pair p, the forward C2C's input.
__global__ void k_fix_to_pairs(unsigned long long* __restrict__ fx, float2* __restrict__ pairs, long long npairs,
                               long long M) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= npairs * M) return;
  const long long p = k / M, m = k - p * M;
  unsigned long long* a = fx + 2 * p * M + m;
  const long long va = (long long)a[0], vb = (long long)a[M];
  pairs[k] = make_float2((float)((double)va * kInvFix), (float)((double)vb * kInvFix));
  a[0] = 0ull;
  a[M] = 0ull;
}

// paired density spectra -> per-channel half spectra (the R2C layout, for the observables and S(k)):
// one thread per half-spectrum point, every pair of the system
__global__ void k_unpack_half(const float2* __restrict__ z, float2* __restrict__ half, int npairs, Geom g, int D) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= g.Mh) return;
  const unsigned hu = (unsigned)h, rr = hu / (unsigned)g.nxh;
  const int ix = (int)(hu - rr * (unsigned)g.nxh), iy = (int)(rr % (unsigned)g.nx[1]), iz = (int)(rr / (unsigned)g.nx[1]);
  const int nx = g.nx[0], ny = g.nx[1], nz = D == 3 ? g.nx[2] : 1;
  const long long fk = ((long long)iz * ny + iy) * nx + ix;
  const long long fmk = ((long long)(iz ? nz - iz : 0) * ny + (iy ? ny - iy : 0)) * nx + (ix ? nx - ix : 0);
  for (int p = 0; p < npairs; p++) {
    const float2 a = z[(long long)p * g.M + fk], am = z[(long long)p * g.M + fmk];
    half[(long long)(2 * p) * g.Mh + h] = pair_unpack(a, am, 0);
    half[(long long)(2 * p + 1) * g.Mh + h] = pair_unpack(a, am, 1);
  }
}

// paired densities -> planar channels (density reads and snapshots): n = pairs x M
__global__ void k_pairs_to_planar(const float2* __restrict__ pairs, float* __restrict__ planar, long long npairs,
                                  long long M) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= npairs * M) return;
  const long long p = k / M, m = k - p * M;
  const float2 v = pairs[k];
  planar[2 * p * M + m] = v.x;
  planar[(2 * p + 1) * M + m] = v.y;
}

// ---------------------------------------------------------------------------------------------
// k-space multiply (replaces d_prepareForceKSpace, device_array_utils.cu:298-312, for every
// style and side, and d_prepareElectrostaticPotential / d_prepareElectricField :199-241)
// ---------------------------------------------------------------------------------------------
template <int D, int NT>
__global__ void __launch_bounds__(256) k_kmul(const float2* __restrict__ rhok_all, float2* __restrict__ gk_all,
                                             const float* __restrict__ utab_all, const float* __restrict__ ctab_all,
                                             const float* __restrict__ kd_all, const int* __restrict__ cta_sys,
                                             const int* __restrict__ blk0, const SysDev* __restrict__ sysd,
                                             int integrate, int blk_off) {
  const int blk = blockIdx.x + blk_off;
  const int s = cta_sys[blk];
  const SysDev& sd = sysd[s];
  if (!sd.active) return;  // one system per CTA; inactive systems are not gathered
  // per-CTA style table: the CTA covers one system
  __shared__ float s_scale[TILD_MAX_STYLES];
  __shared__ int s_ab[TILD_MAX_STYLES];
  __shared__ int s_nfft;
  const long long est = sd.step + (integrate ? 1 : 0);
  if (threadIdx.x < TILD_MAX_STYLES && threadIdx.x < sd.nfft) {
    s_scale[threadIdx.x] = ramp_ratio(sd, threadIdx.x, est);
    s_ab[threadIdx.x] = sd.sa[threadIdx.x] | (sd.sb[threadIdx.x] << 8);
  }
  if (threadIdx.x == 0) s_nfft = sd.nfft;
  __syncthreads();
  const Geom& g = sd.g;
  const long long h = (long long)(blk - blk0[s]) * blockDim.x + threadIdx.x;
  const long long Mh = g.Mh;
  if (h >= Mh) return;
  const int T = sd.T, C = sd.C;
  const int nfft = s_nfft;
  const float* utab = utab_all + sd.utab0 + h;
  const float2* rhok = rhok_all + sd.spec0;
  const float* kd = kd_all + sd.kd0;
  // 32-bit index arithmetic: grids hold fewer than 2^31 points (tild_create checks)
  const unsigned hu = (unsigned)h, rr = hu / (unsigned)g.nxh;
  const int ix = (int)(hu - rr * (unsigned)g.nxh);
  const int iy = (int)(rr % (unsigned)g.nx[1]);
  const int iz = (int)(rr / (unsigned)g.nx[1]);
  float kv[3];
  kv[0] = kd[ix];
  kv[1] = kd[g.nx[0] + iy];
  kv[2] = (D == 3) ? kd[g.nx[0] + g.nx[1] + iz] : 0.f;
  // output: -i k_d P for each channel's potential P, planar per direction (batched C2R input); or,
  // with inv_packed, W = G_a + i G_b for each channel pair (a, b) = (2p, 2p + 1) over the full
  // spectrum (batched C2C input): W(k) here, and W(-k) = conj(G_a) + i conj(G_b) when -k lies
  // outside the half spectrum (0 < ix < nx/2), so the complex inverse returns g_a + i g_b
  const bool packed = sd.inv_packed, fwd = sd.fwd_packed;
  float2* gk = packed ? gk_all + sd.gkp0 : gk_all + sd.spec0 * D;
  long long fk = 0, fmk = 0;  // full-spectrum indices of k and -k
  bool mirror = false;
  if (packed || fwd) {
    const int nx = g.nx[0], ny = g.nx[1], nz = D == 3 ? g.nx[2] : 1;
    fk = ((long long)iz * ny + iy) * nx + ix;
    fmk = ((long long)(iz ? nz - iz : 0) * ny + (iy ? ny - iy : 0)) * nx + (ix ? nx - ix : 0);
    mirror = ix > 0 && 2 * ix != nx;
  }
  const long long M = g.M;
  // a channel's density spectrum at k: the R2C output, or, with fwd_packed, from its pair's
  // spectrum Z = X_2p + i X_2p+1: X_2p = (Z(k) + conj Z(-k)) / 2, X_2p+1 = (Z(k) - conj Z(-k)) / 2i
  const float2* zpairs = rhok_all + sd.rkp0;
  auto rho_hat = [&](int ch) -> float2 {
    if (!fwd) return rhok[(long long)ch * Mh + h];
    const float2* zp = zpairs + (long long)(ch >> 1) * M;
    return pair_unpack(zp[fk], zp[fmk], ch & 1);
  };
  float2 held = make_float2(0.f, 0.f);
  auto store = [&](int ch, float2 P) {
    if (!packed) {
#pragma unroll
      for (int d = 0; d < D; d++) gk[((long long)ch * D + d) * Mh + h] = make_float2(kv[d] * P.y, -kv[d] * P.x);
      return;
    }
    if (!(ch & 1)) {  // channels come in order; the pair is written with its odd channel
      held = P;
      return;
    }
    float2* W = gk + (long long)(ch >> 1) * D * M;
#pragma unroll
    for (int d = 0; d < D; d++) {
      const float2 ga = make_float2(kv[d] * held.y, -kv[d] * held.x);
      const float2 gb = make_float2(kv[d] * P.y, -kv[d] * P.x);
      W[d * M + fk] = make_float2(ga.x - gb.y, ga.y + gb.x);
      if (mirror) W[d * M + fmk] = make_float2(ga.x + gb.y, gb.x - ga.y);
    }
  };
  if (NT > 0) {
    constexpr int NA = NT > 0 ? NT : 1;
    float2 rk[NA], phi[NA];
#pragma unroll
    for (int t = 0; t < NA; t++) {
      rk[t] = (t < T) ? rho_hat(t) : make_float2(0.f, 0.f);
      phi[t] = make_float2(0.f, 0.f);
    }
    for (int k = 0; k < nfft; k++) {
      const float u = utab[(long long)k * Mh] * s_scale[k];
      const int a = s_ab[k] & 0xff, b = s_ab[k] >> 8;
      // explicit selects keep rk[] and phi[] in registers
      float2 ra = make_float2(0.f, 0.f), rb = make_float2(0.f, 0.f);
#pragma unroll
      for (int t = 0; t < NA; t++) {
        if (t == a) ra = rk[t];
        if (t == b) rb = rk[t];
      }
#pragma unroll
      for (int t = 0; t < NA; t++) {
        if (t == a) { phi[t].x += u * rb.x; phi[t].y += u * rb.y; }
        if (t == b) { phi[t].x += u * ra.x; phi[t].y += u * ra.y; }
      }
    }
#pragma unroll
    for (int t = 0; t < NA; t++) {
      if (t >= T) break;
      store(t, phi[t]);
    }
  } else {  // more types than the specialised kernels cover: same arithmetic, local arrays
    float2 phi[TILD_MAX_TYPES];
    for (int t = 0; t < T; t++) phi[t] = make_float2(0.f, 0.f);
    for (int k = 0; k < nfft; k++) {
      const float u = utab[(long long)k * Mh] * s_scale[k];
      const int a = s_ab[k] & 0xff, b = s_ab[k] >> 8;
      const float2 ra = rho_hat(a), rb = rho_hat(b);
      phi[a].x += u * rb.x; phi[a].y += u * rb.y;
      phi[b].x += u * ra.x; phi[b].y += u * ra.y;
    }
    for (int t = 0; t < T; t++) store(t, phi[t]);
  }
  if (C) {
    const float2 rc = rho_hat(T);
    const float cm = ctab_all[sd.ctab0 + h];
    const float2 pc = make_float2(cm * rc.x, cm * rc.y);
    store(T, pc);
  }
}

// fieldphase: gather field of type a gets +rho_a f_r, of type b gets -rho_b f_r
__global__ void k_fieldphase_apply(float* __restrict__ gfield, const float* __restrict__ rho,
                                   const float* __restrict__ fr, int a, int b, int D, long long M) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= M) return;
  const float ra = rho[(long long)a * M + r], rb = rho[(long long)b * M + r];
  for (int d = 0; d < D; d++) {
    const float f = fr[(long long)d * M + r];
    gfield[((long long)a * D + d) * M + r] += ra * f;
    gfield[((long long)b * D + d) * M + r] -= rb * f;
  }
}

// Interleave the C2R output [(T+C)][D][M] into one float4 (-dPhi/dx, -dPhi/dy, -dPhi/dz, 0) per
// grid point and channel, so the gather reads a stencil node with a single 16-byte load.
// (Writing the float4 field from strided inverse transforms instead was measured slower at 128^3
// and no faster on small grids.)
template <int D>
__global__ void k_interleave(const float* __restrict__ planar_all, const float2* __restrict__ pairs_all,
                             float4* __restrict__ g4_all, const int* __restrict__ cta_sys, const int* __restrict__ blk0,
                             const SysDev* __restrict__ sysd, int layout, int blk_off) {
  const int blk = blockIdx.x + blk_off;
  const int s = cta_sys[blk];
  const SysDev& sd = sysd[s];
  if (!sd.active) return;  // inactive systems are not gathered
  const Geom& g = sd.g;
  const long long M = g.M;
  const long long m = (long long)(blk - blk0[s]) * blockDim.x + threadIdx.x;
  if (m >= M) return;
  long long dst = m;
  if (layout != TILD_FIELD_LINEAR) {  // 32-bit index arithmetic: grids hold fewer than 2^31 points
    const unsigned mu = (unsigned)m, r = mu / (unsigned)g.nx[0];
    const int x = (int)(mu - r * (unsigned)g.nx[0]);
    const int y = (int)(r % (unsigned)g.nx[1]), z = (int)(r / (unsigned)g.nx[1]);
    dst = tild_field_off(layout, 0, x, g) + tild_field_off(layout, 1, y, g) + tild_field_off(layout, 2, z, g);
  }
  const float* planar = planar_all + sd.grid0 * D;
  float4* g4 = g4_all + sd.g4_0;
  const int nch = sd.T + sd.C;
  if (sd.inv_packed) {  // pair p's direction d is one complex field: real part channel 2p, imaginary 2p + 1
    const float2* z = pairs_all + sd.gkp0;
    for (int p = 0; p < nch / 2; p++) {
      const float2* src = z + (long long)p * D * M + m;
      const float2 vx = src[0], vy = src[M], vz = D == 3 ? src[2 * M] : make_float2(0.f, 0.f);
      g4[(long long)(2 * p) * sd.Mb + dst] = make_float4(vx.x, vy.x, vz.x, 0.f);
      g4[(long long)(2 * p + 1) * sd.Mb + dst] = make_float4(vx.y, vy.y, vz.y, 0.f);
    }
    return;
  }
  for (int ch = 0; ch < nch; ch++) {
    const float* src = planar + (long long)ch * D * M + m;
    g4[(long long)ch * sd.Mb + dst] = make_float4(src[0], src[M], D == 3 ? src[2 * M] : 0.f, 0.f);
  }
}

// ---------------------------------------------------------------------------------------------
// Gather + bonds + integrators (d_add_grid_forces{2D,3D}, d_add_grid_forces_charges_*,
// device_grid_utils.cu:346-452; d_bonds, device_bonds.cu:4-60; d_GJF_integrator,
// device_GJF_integrator.cu:4-62; d_EM_integrator, device_EM_integrator.cu:5-36)
// ---------------------------------------------------------------------------------------------
template <int D, int P>
__device__ __forceinline__ void gather4(const float4* __restrict__ F, const float (&W)[3][P + 1],
                                        const int (&o)[3][P + 1], float (&acc)[3]) {
#pragma unroll
  for (int ix = 0; ix <= P; ix++)
#pragma unroll
    for (int iy = 0; iy <= P; iy++) {
      const float wxy = W[0][ix] * W[1][iy];
      const int row = o[0][ix] + o[1][iy];
      if (D == 3) {
#pragma unroll
        for (int iz = 0; iz <= P; iz++) {
          const float4 v = __ldg(F + row + o[2][iz]);
          const float w = wxy * W[2][iz];
          acc[0] += v.x * w;
          acc[1] += v.y * w;
          acc[2] += v.z * w;
        }
      } else {
        const float4 v = __ldg(F + row);
        acc[0] += v.x * wxy;
        acc[1] += v.y * wxy;
      }
    }
}

// Order 3 in 3D: the 64-node sum is split into 8 partial sums, one per (x column ix, row parity
// pr), each over rows iy = pr, pr + 2 and the 4 z nodes in that order, combined by a fixed tree.
// The quarter-warp gather below computes exactly this association with one lane per partial
// (8 lanes per bead); every other order-3 3D path uses the same helpers, so all of them give the
// same bits.
__device__ __forceinline__ void p3_node(const float4& v, float w, float (&a)[3]) {
  a[0] = __fmaf_rn(v.x, w, a[0]);
  a[1] = __fmaf_rn(v.y, w, a[1]);
  a[2] = __fmaf_rn(v.z, w, a[2]);
}
// a charge channel joins the type channel's sum as F + E q
__device__ __forceinline__ float p3_join_charge(float f, float e, float q) { return __fmaf_rn(e, q, f); }

// One thread's order-3 3D sum in that association; ld(ix, iy, iz) returns the node.
template <class Ld>
__device__ __forceinline__ void p3_partial(const float (&W)[3][4], Ld ld, int ix, int pr, float (&a)[3]) {
  a[0] = a[1] = a[2] = 0.f;
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const int iy = pr + 2 * k;
    const float wxy = W[0][ix] * W[1][iy];
#pragma unroll
    for (int iz = 0; iz < 4; iz++) p3_node(ld(ix, iy, iz), wxy * W[2][iz], a);
  }
}
// The tree over partials s_l, l = ix + 4 pr: ((s0 + s1) + (s2 + s3)) + ((s4 + s5) + (s6 + s7)),
// each pair added as soon as it exists (fewer live registers).
template <class Ld>
__device__ __forceinline__ void p3_sum_sequential(const float (&W)[3][4], Ld ld, float (&acc)[3]) {
  float u[2][3];
#pragma unroll
  for (int pr = 0; pr < 2; pr++) {
    float t[2][3];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      float a[3], b[3];
      p3_partial(W, ld, 2 * h, pr, a);
      p3_partial(W, ld, 2 * h + 1, pr, b);
#pragma unroll
      for (int d = 0; d < 3; d++) t[h][d] = __fadd_rn(a[d], b[d]);
    }
#pragma unroll
    for (int d = 0; d < 3; d++) u[pr][d] = __fadd_rn(t[0][d], t[1][d]);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) acc[d] = __fadd_rn(u[0][d], u[1][d]);
}

// The order-3 3D stencil of a warp's 32 slots, 8 lanes per bead.  A request of 8 lanes reads one
// bead's 4 x-neighbour nodes in two adjacent rows: 8 distinct 16-byte bank groups in the brick
// and linear field layouts, so every stencil request costs the 4 L1 data wavefronts of its
// quarters (with a bead per lane the quarters' beads collide in banks: 7.6 wavefronts per request
// on the sorted blend, 10 once the sort is stale).  Each lane first stages its own bead's
// weights and node offsets in shared memory; in round r quarter q sums bead 8q + r (lane
// ix + 4 pr taking partial (ix, pr)), reduces over its 8 lanes with three xor-shuffles, and the
// bead's own lane (8q + r) keeps the total.  Invalid slots stage offset -1 and are skipped by
// their quarter.  Every lane of the warp must call it.
template <bool CH>
__device__ __forceinline__ void p3_quarter_stencil(bool valid, const int (&o)[3][4], const float (&W)[3][4],
                                                   int tch, int qch, float q, const float4* __restrict__ F,
                                                   float (&f)[3]) {
  __shared__ float2 sX[kTile * 4];   // {Wx[ix], x offset + type channel}, bead slots paired by bit 3
  __shared__ float4 sY[kTile * 2];   // {Wy[pr], Wy[pr + 2], y offsets of rows pr and pr + 2}
  __shared__ float4 sWz[kTile];
  __shared__ int4 sOz[kTile];
  __shared__ float2 sQ[CH ? kTile : 1];  // {q, offset from the type channel to the charge channel}
  const int tid = threadIdx.x, lane = tid & 31, wb = tid & ~31;
  {
    const int js = wb | ((lane ^ ((lane >> 3) & 1)) & 31);  // beads j and j + 8 of a half-warp: other banks
#pragma unroll
    for (int ix = 0; ix < 4; ix++)
      sX[js * 4 + ix] = make_float2(W[0][ix], __int_as_float(valid ? o[0][ix] + tch : -1));
#pragma unroll
    for (int pr = 0; pr < 2; pr++)
      sY[tid * 2 + pr] = make_float4(W[1][pr], W[1][pr + 2], __int_as_float(o[1][pr]), __int_as_float(o[1][pr + 2]));
    sWz[tid] = make_float4(W[2][0], W[2][1], W[2][2], W[2][3]);
    sOz[tid] = make_int4(o[2][0], o[2][1], o[2][2], o[2][3]);
    if (CH) sQ[tid] = make_float2(valid ? q : 0.f, __int_as_float(qch - tch));
  }
  __syncwarp();
  const int qt = lane >> 3, l8 = lane & 7, ix = l8 & 3, pr = l8 >> 2;
#pragma unroll 1
  for (int r = 0; r < 8; r++) {
    const int jw = 8 * qt + r;  // bead of this quarter, within the warp
    const int j = wb | jw;
    const float2 xv = sX[(wb | (jw ^ ((jw >> 3) & 1))) * 4 + ix];
    const int ox = __float_as_int(xv.y);
    float a[3] = {0.f, 0.f, 0.f}, e[3] = {0.f, 0.f, 0.f};
    float qj = 0.f;
    if (ox >= 0) {  // the same for the quarter's 8 lanes
      const float4 yv = sY[j * 2 + pr];
      const float4 wz = sWz[j];
      const int4 oz = sOz[j];
      const float wy[2] = {yv.x, yv.y};
      const int oy[2] = {__float_as_int(yv.z), __float_as_int(yv.w)};
      const float wzv[4] = {wz.x, wz.y, wz.z, wz.w};
      const int ozv[4] = {oz.x, oz.y, oz.z, oz.w};
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const float wxy = xv.x * wy[k];
        const float4* row = F + (ox + oy[k]);
#pragma unroll
        for (int iz = 0; iz < 4; iz++) p3_node(__ldg(row + ozv[iz]), wxy * wzv[iz], a);
      }
      if (CH) {
        const float2 qv = sQ[j];
        qj = qv.x;
        if (qj != 0.f) {
          const int dq = __float_as_int(qv.y);
#pragma unroll
          for (int k = 0; k < 2; k++) {
            const float wxy = xv.x * wy[k];
            const float4* row = F + (ox + dq + oy[k]);
#pragma unroll
            for (int iz = 0; iz < 4; iz++) p3_node(__ldg(row + ozv[iz]), wxy * wzv[iz], e);
          }
        }
      }
    }
    // s_l + s_(l^1), then pairs, then quads: p3_sum_sequential's tree, on every lane of the quarter
#pragma unroll
    for (int m = 1; m <= 4; m <<= 1)
#pragma unroll
      for (int d = 0; d < 3; d++) {
        a[d] = __fadd_rn(a[d], __shfl_xor_sync(0xffffffffu, a[d], m));
        if (CH) e[d] = __fadd_rn(e[d], __shfl_xor_sync(0xffffffffu, e[d], m));
      }
    if (l8 == r) {
#pragma unroll
      for (int d = 0; d < 3; d++) f[d] = CH && qj != 0.f ? p3_join_charge(a[d], e[d], qj) : a[d];
    }
  }
}

// stencil node indices -> offsets in one channel of the force field
template <int D, int P>
__device__ __forceinline__ void field_offsets(const int (&idx)[3][P + 1], int layout, const Geom& g,
                                              int (&o)[3][P + 1]) {
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int a = 0; a <= P; a++) o[d][a] = d < D ? tild_field_off(layout, d, idx[d][a], g) : 0;
}

// Bonds, the force output and the integrators of one bead: d_bonds (device_bonds.cu:4-60) and
// Integrate_2 (integrator.cu:24-39) over the integrators in input order.  Shared by both gathers.
template <int D, bool INTEG, bool XW>
__device__ __forceinline__ void bead_epilogue(int i, const float4& p, int t, float (&x)[3], float (&f)[3],
                                              const SysDev& sd, const Geom& g, int info, int nb,
                                              const float4 (&pj)[3], int bid, const float4& po,
                                              float* __restrict__ noise, float4* __restrict__ pos_io,
                                              float* __restrict__ f_out, int f_sys, int s,
                                              curandStateXORWOW_t* __restrict__ xw) {
  // bonds
#pragma unroll
  for (int bb = 0; bb < 3; bb++) {
    if (bb >= nb) break;
    const int bt = (info >> (8 + 8 * bb)) & 0xff;
    const float xj[3] = {pj[bb].x, pj[bb].y, pj[bb].z};
    float dr[3], mdr2 = 0.f;
#pragma unroll
    for (int d = 0; d < D; d++) {
      dr[d] = x[d] - xj[d];
      if (dr[d] > g.Lh[d]) dr[d] -= g.L[d];
      else if (dr[d] < -g.Lh[d]) dr[d] += g.L[d];
      mdr2 += dr[d] * dr[d];
    }
    float mf = 0.f;
    if (mdr2 > 1.0E-4f) {
      const float mdr = sqrtf(mdr2);
      mf = 2.0f * sd.bond_k[bt] * (mdr - sd.bond_req[bt]) / mdr;
    }
#pragma unroll
    for (int d = 0; d < D; d++) f[d] -= mf * dr[d];
  }
  if (f_out && s == f_sys) {
#pragma unroll
    for (int d = 0; d < D; d++) f_out[(long long)bid * D + d] = f[d];
  }
  if (!INTEG) return;
  // integrators in input order (integrator.cu:24-39 is called for each in turn)
  const int mask = sd.type_mask[t];
  const long long est = sd.step + 1;
  float xo[3] = {po.x, po.y, po.z};
  float on[3] = {0.f, 0.f, 0.f};
  bool any_gjf = false;
  curandStateXORWOW_t st;
  if (XW && mask) st = xw[i];
  for (int ig = 0; ig < sd.n_integ; ig++) {
    if (!(mask & (1 << ig))) continue;
    float z[3];
    if (XW) {
#pragma unroll
      for (int d = 0; d < D; d++) z[d] = curand_normal(&st);
    } else {
      philox_normal3(sd.seed, (uint32_t)bid, est, (uint32_t)ig, z);
    }
    if (sd.integ_kind[ig] == TILD_INTEGRATOR_GJF) {
      if (!any_gjf) {
#pragma unroll
        for (int d = 0; d < D; d++) on[d] = noise[3 * (long long)i + d];
        any_gjf = true;
      }
      const float m = sd.mass[t], df = sd.diff[t], delt = sd.delt;
      const float b = m / (m + delt / (2.0f * df));
      const float a = (1.0f - delt / (2.0f * df * m)) / (1.0f + delt / (2.0f * df * m));
      const float delt2 = delt * delt;
#pragma unroll
      for (int d = 0; d < D; d++) {
        const float nn = sd.noise_mag / df * z[d];
        const float xtmp = x[d];
        if (xo[d] - x[d] > g.L[d] / 2.0f) xo[d] -= g.L[d];
        else if (xo[d] - x[d] < -g.L[d] / 2.0f) xo[d] += g.L[d];
        float xn = 2.0f * b * x[d] - a * xo[d] + b * delt2 / m * f[d] + b * delt / (2.0f * m) * (nn + on[d]);
        xo[d] = xtmp;
        on[d] = nn;
        if (xn > g.L[d]) xn -= g.L[d];
        else if (xn < 0.0f) xn += g.L[d];
        x[d] = xn;
      }
    } else {
#pragma unroll
      for (int d = 0; d < D; d++) {
        float xn = x[d] + sd.delt * f[d] + sd.noise_mag * z[d];
        if (xn > g.L[d]) xn -= g.L[d];
        else if (xn < 0.0) xn += g.L[d];
        x[d] = xn;
      }
    }
  }
  if (XW && mask) xw[i] = st;
  pos_io[i] = make_float4(x[0], x[1], D == 3 ? x[2] : 0.f, p.w);
  if (any_gjf) {
#pragma unroll
    for (int d = 0; d < D; d++) noise[3 * (long long)i + d] = on[d];
  }
}

// SPR (integrating launches only): after the update the kernel spreads x_{n+1} into the density
// accumulator for the next step, through the shared box (1) or the global atomics (2), so the
// next step needs no spread kernel.  Inactive systems spread their held positions.  The integer
// sums are those of the spread kernel, bitwise.
template <int D, int P, bool INTEG, bool XW, bool CH, int SPR>
__global__ void __launch_bounds__(256, (P >= 4 ? 2 : (P >= 3 ? 4 : (P >= 2 ? 3 : 4)))) k_gather(
    const float4* __restrict__ pos_in, float4* __restrict__ pos_io, float* __restrict__ noise,
    const int* __restrict__ bead_id, const int* __restrict__ bond_nbr, const int* __restrict__ bond_info,
    const float* __restrict__ charge, const float4* __restrict__ g4_all, const int* __restrict__ cta_sys,
    const SysDev* __restrict__ sysd, float* __restrict__ f_out, int f_sys, curandStateXORWOW_t* __restrict__ xw,
    int layout, unsigned long long* __restrict__ rho_fx_all, int spread_cap, int* status, int blk_off) {
  static_assert(SPR == 0 || INTEG, "only integrating launches spread ahead");
  const int s = cta_sys[blockIdx.x + blk_off];
  const SysDev& sd = sysd[s];
  const int i = (blockIdx.x + blk_off) * blockDim.x + threadIdx.x;
  const float4 p = pos_in[i];
  const int t = tild_type_of(p.w);
  float x[3] = {p.x, p.y, p.z};
  const bool finite = isfinite(p.x) && isfinite(p.y) && (D == 2 || isfinite(p.z));
  const int C = sd.C;
  const float q = (CH && C && t != kPadType) ? charge[i] : 0.f;
  bool sp = false;  // x (after the update) is spread ahead
  if (!sd.active) {  // one system per CTA: every thread takes this branch together
    if (INTEG) pos_io[i] = p;  // inactive systems keep x_n through the buffer rotation
    if (SPR == 0) return;
    sp = t != kPadType && finite;  // held positions are spread too
    if (t != kPadType && !finite) atomicOr(status, ST_NONFINITE_POS);
  } else if constexpr (D == 3 && P == 3) {
    // the quarter-warp stencil needs every lane of the warp, valid slot or not
    const bool valid = t != kPadType && finite;
    if (t != kPadType && !finite) atomicOr(status, ST_NONFINITE_POS);
    const Geom& g = sd.g;
    float W[3][4] = {};
    int o[3][4] = {};
    if (valid) {
      int idx[3][4];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int b = axis_base<3>(x[d], g.dx[d], W[d]);
#pragma unroll
        for (int a = 0; a <= 3; a++) idx[d][a] = wrap_idx(b + a, g.nx[d], status);
      }
      field_offsets<3, 3>(idx, layout, g, o);
    }
    const long long Mb = sd.Mb;
    float f[3] = {0.f, 0.f, 0.f};
    p3_quarter_stencil<CH>(valid, o, W, valid ? (int)(t * Mb) : 0, (int)(sd.T * Mb), q, g4_all + sd.g4_0, f);
    if (!valid) {
      if (SPR == 0) return;
    } else {
      const int info = bond_info[i];
      const int nb = info & 3;
      float4 pj[3];
#pragma unroll
      for (int bb = 0; bb < 3; bb++)
        if (bb < nb) pj[bb] = pos_in[bond_nbr[3 * i + bb]];
      const int bid = bead_id[i];
      float4 po = make_float4(0.f, 0.f, 0.f, 0.f);
      if (INTEG) po = pos_io[i];
      bead_epilogue<D, INTEG, XW>(i, p, t, x, f, sd, g, info, nb, pj, bid, po, noise, pos_io, f_out, f_sys, s, xw);
      if (SPR != 0) {
        sp = isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]);
        if (!sp) atomicOr(status, ST_NONFINITE_POS);
      }
    }
  } else if (t != kPadType && !finite) {
    atomicOr(status, ST_NONFINITE_POS);
    if (SPR == 0) return;  // left in place; the host reports TILD_ERR_NAN
  } else if (t != kPadType) {
    const Geom& g = sd.g;
    const long long Mb = sd.Mb;
    const int T = sd.T;
    const float4* g4 = g4_all + sd.g4_0;

    float f[3] = {0.f, 0.f, 0.f};
    {
      float W[3][P + 1];
      int idx[3][P + 1];
#pragma unroll
      for (int d = 0; d < D; d++) {
        const int b = axis_base<P>(x[d], g.dx[d], W[d]);
#pragma unroll
        for (int a = 0; a <= P; a++) idx[d][a] = wrap_idx(b + a, g.nx[d], status);
      }
      int o[3][P + 1];
      field_offsets<D, P>(idx, layout, g, o);
      if (CH && C && q != 0.f) {
        float e[3] = {0.f, 0.f, 0.f};
        gather4<D, P>(g4 + (long long)T * Mb, W, o, e);
#pragma unroll
        for (int d = 0; d < D; d++) f[d] += e[d] * q;
      }
      gather4<D, P>(g4 + (long long)t * Mb, W, o, f);
    }
    // bond partners and x_{n-1} are read after the stencil: held across it they cost the stencil
    // registers (measured 1-4 % slower gathers)
    const int info = bond_info[i];
    const int nb = info & 3;
    float4 pj[3];
#pragma unroll
    for (int bb = 0; bb < 3; bb++)
      if (bb < nb) pj[bb] = pos_in[bond_nbr[3 * i + bb]];
    const int bid = bead_id[i];
    float4 po = make_float4(0.f, 0.f, 0.f, 0.f);
    if (INTEG) po = pos_io[i];  // x_{n-1} (GJF xo)
    bead_epilogue<D, INTEG, XW>(i, p, t, x, f, sd, g, info, nb, pj, bid, po, noise, pos_io, f_out, f_sys, s, xw);
    if (SPR != 0) {
      sp = isfinite(x[0]) && isfinite(x[1]) && (D == 2 || isfinite(x[2]));
      if (!sp) atomicOr(status, ST_NONFINITE_POS);
    }
  } else if (SPR == 0) {
    return;  // padding slot
  }
  if constexpr (SPR == 1) cta_spread_box<D, P, CH>(sp, x, t, q, sd, rho_fx_all + sd.grid0, spread_cap, status);
  if constexpr (SPR == 2)
    if (sp) bead_spread_direct<D, P, CH>(x, t, q, sd, rho_fx_all);
}

// The same stencil sums read from a shared-memory box: the CTA's 256 slots (spatially sorted, so
// a few bricks of cells) need a box of roughly 11x11x7 nodes per channel at order 3.  The box is
// loaded once with coalesced rows, then every bead reads its (P+1)^D nodes from shared memory in
// the gather4 order, so forces are bitwise those of k_gather.  A chunk whose box does not fit
// reads global memory like k_gather.
template <int D, int P>
__device__ __forceinline__ void box_gather4(const float4* __restrict__ B, const float (&W)[3][P + 1],
                                            const int (&lb)[3], int ex, int exy, float (&acc)[3]) {
#pragma unroll
  for (int ix = 0; ix <= P; ix++)
#pragma unroll
    for (int iy = 0; iy <= P; iy++) {
      const float wxy = W[0][ix] * W[1][iy];
      const int row = (lb[1] + iy) * ex + lb[0] + ix;
      if (D == 3) {
#pragma unroll
        for (int iz = 0; iz <= P; iz++) {
          const float4 v = B[row + (lb[2] + iz) * exy];
          const float w = wxy * W[2][iz];
          acc[0] += v.x * w;
          acc[1] += v.y * w;
          acc[2] += v.z * w;
        }
      } else {
        const float4 v = B[row];
        acc[0] += v.x * wxy;
        acc[1] += v.y * wxy;
      }
    }
}

template <int D, int P, bool INTEG, bool XW, bool CH>
__global__ void __launch_bounds__(256, (P >= 4 ? 2 : 3)) k_gather_box(
    const float4* __restrict__ pos_in, float4* __restrict__ pos_io, float* __restrict__ noise,
    const int* __restrict__ bead_id, const int* __restrict__ bond_nbr, const int* __restrict__ bond_info,
    const float* __restrict__ charge, const float4* __restrict__ g4_all, const int* __restrict__ cta_sys,
    const SysDev* __restrict__ sysd, float* __restrict__ f_out, int f_sys, curandStateXORWOW_t* __restrict__ xw,
    int box_cap, int* status, int blk_off) {
  extern __shared__ float4 sbox[];
  __shared__ int s_g0[3], s_min[3], s_max[3];
  __shared__ int s_row[kMaxRows];
  const int s = cta_sys[blockIdx.x + blk_off];
  const SysDev& sd = sysd[s];
  const int i0 = (blockIdx.x + blk_off) * blockDim.x;
  const int i = i0 + threadIdx.x;
  if (!sd.active) {  // one system per CTA: every thread leaves here together
    if (INTEG) pos_io[i] = pos_in[i];
    return;
  }
  const Geom g = sd.g;
  chunk_origin<D, P>(pos_in, i0, g, s_g0, s_min, s_max);
  const float4 p = pos_in[i];
  const int t = tild_type_of(p.w);
  float x[3] = {p.x, p.y, p.z};
  bool ok = t != kPadType;
  if (ok && !(isfinite(p.x) && isfinite(p.y) && (D == 2 || isfinite(p.z)))) {
    atomicOr(status, ST_NONFINITE_POS);
    ok = false;  // left in place; the host reports TILD_ERR_NAN
  }
  float W[3][P + 1];
  int rel[3] = {0, 0, 0}, base[3] = {0, 0, 0};
  if (ok) {
#pragma unroll
    for (int d = 0; d < D; d++) {
      base[d] = axis_base<P>(x[d], g.dx[d], W[d]);
      if (base[d] < -g.nx[d] || base[d] + P >= 2 * g.nx[d]) atomicOr(status, ST_INDEX_RANGE);
      rel[d] = fold_rel(base[d] - s_g0[d], g.nx[d]);
    }
  }
  int info = 0, nb = 0, bid = 0;
  float4 pj[3];
  float4 po = make_float4(0.f, 0.f, 0.f, 0.f);
  if (ok) {
    info = bond_info[i];
    nb = info & 3;
#pragma unroll
    for (int bb = 0; bb < 3; bb++)
      if (bb < nb) pj[bb] = pos_in[bond_nbr[3 * i + bb]];
    bid = bead_id[i];
    if (INTEG) po = pos_io[i];
  }
  int mn[3], ext[3];
  long long vol;
  if (!chunk_box<D, P>(ok, rel, s_min, s_max, mn, ext, vol)) return;
  const long long Mb = sd.Mb;  // the box gather runs on the linear layout
  const int T = sd.T, C = sd.C, nch = T + C;
  const float4* g4 = g4_all + sd.g4_0;
  const float q = (CH && C && ok) ? charge[i] : 0.f;
  float f[3] = {0.f, 0.f, 0.f};
  const int ex = ext[0], ey = ext[1], ez = ext[2];
  if (vol * nch <= box_cap && ex <= 64 && ey * ez <= kMaxRows) {
    // row offsets of the box in the periodic grid, then the rows themselves, lanes along x
    const int rows = ey * ez;
    for (int yz = threadIdx.x; yz < rows; yz += blockDim.x) {
      const int ly = yz % ey, lz = yz / ey;
      s_row[yz] = (int)((long long)g.nx[0] * (pmod(s_g0[1] + mn[1] + ly, g.nx[1]) +
                                              (long long)g.nx[1] * (D == 3 ? pmod(s_g0[2] + mn[2] + lz, g.nx[2]) : 0)));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int lpr = ex < 32 ? ex : 32;           // lanes per row
    const int rpi = 32 / lpr;                    // rows per warp iteration
    const int my_r = lane / lpr, my_x = lane - my_r * lpr;
    const int bx = pmod(s_g0[0] + mn[0], g.nx[0]);
    int xo[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
      int xg = bx + my_x + 32 * k;
      if (xg >= g.nx[0]) xg -= g.nx[0];
      if (xg >= g.nx[0]) xg %= g.nx[0];
      xo[k] = xg;
    }
    const int nrows = rows * nch;
    if (my_r < rpi)
      for (int R = warp * rpi + my_r; R < nrows; R += nwarps * rpi) {
        const int ch = R / rows, yz = R - ch * rows;
        const float4* src = g4 + (long long)ch * Mb + s_row[yz];
        float4* dst = sbox + (long long)ch * vol + (long long)yz * ex;
#pragma unroll
        for (int k = 0; k < 2; k++) {
          const int lx = my_x + 32 * k;
          if (lx < ex) dst[lx] = __ldg(src + xo[k]);
        }
      }
    __syncthreads();
    if (ok) {
      int lb[3] = {0, 0, 0};
#pragma unroll
      for (int d = 0; d < D; d++) lb[d] = rel[d] - mn[d];
      if constexpr (D == 3 && P == 3) {  // the association of the quarter-warp gather
        const int exy = ex * ey;
        const float4* bt = sbox + (long long)t * vol;
        p3_sum_sequential(W, [&](int ix, int iy, int iz) { return bt[(lb[2] + iz) * exy + (lb[1] + iy) * ex + lb[0] + ix]; }, f);
        if (CH && C && q != 0.f) {
          const float4* bq = sbox + (long long)T * vol;
          float e[3];
          p3_sum_sequential(W, [&](int ix, int iy, int iz) { return bq[(lb[2] + iz) * exy + (lb[1] + iy) * ex + lb[0] + ix]; }, e);
#pragma unroll
          for (int d = 0; d < 3; d++) f[d] = p3_join_charge(f[d], e[d], q);
        }
      } else {
        if (CH && C && q != 0.f) {
          float e[3] = {0.f, 0.f, 0.f};
          box_gather4<D, P>(sbox + (long long)T * vol, W, lb, ex, ex * ey, e);
#pragma unroll
          for (int d = 0; d < D; d++) f[d] += e[d] * q;
        }
        box_gather4<D, P>(sbox + (long long)t * vol, W, lb, ex, ex * ey, f);
      }
    }
  } else if (ok) {
    int idx[3][P + 1];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int a = 0; a <= P; a++) idx[d][a] = pmod(base[d] + a, g.nx[d]);
    int o[3][P + 1];
    field_offsets<D, P>(idx, TILD_FIELD_LINEAR, g, o);
    if constexpr (D == 3 && P == 3) {
      const float4* ft = g4 + (long long)t * Mb;
      p3_sum_sequential(W, [&](int ix, int iy, int iz) { return __ldg(ft + o[0][ix] + o[1][iy] + o[2][iz]); }, f);
      if (CH && C && q != 0.f) {
        const float4* fq = g4 + (long long)T * Mb;
        float e[3];
        p3_sum_sequential(W, [&](int ix, int iy, int iz) { return __ldg(fq + o[0][ix] + o[1][iy] + o[2][iz]); }, e);
#pragma unroll
        for (int d = 0; d < 3; d++) f[d] = p3_join_charge(f[d], e[d], q);
      }
    } else {
      if (CH && C && q != 0.f) {
        float e[3] = {0.f, 0.f, 0.f};
        gather4<D, P>(g4 + (long long)T * Mb, W, o, e);
#pragma unroll
        for (int d = 0; d < D; d++) f[d] += e[d] * q;
      }
      gather4<D, P>(g4 + (long long)t * Mb, W, o, f);
    }
  }
  if (!ok) return;
  bead_epilogue<D, INTEG, XW>(i, p, t, x, f, sd, g, info, nb, pj, bid, po, noise, pos_io, f_out, f_sys, s, xw);
}

// step counters advance on the device; a system whose counter reaches its stop step leaves the
// active set here, so the next launches skip it without the host in the loop
__global__ void k_advance_steps(SysDev* __restrict__ sysd, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || !sysd[s].active) return;
  const long long step = sysd[s].step + 1;
  sysd[s].step = step;
  if (sysd[s].stop_at >= 0 && step >= sysd[s].stop_at) sysd[s].active = 0;
}

// Order <= 1 always spreads directly; order >= 2 uses the shared box unless the tuner chose the
// direct kernel.  The box (spread_cap words, at most 12288 = 48 KB) plus the kernel's static
// shared memory exceeds the default 48 KB, so the opt-in limit is raised once per device.
// particle blocks [off, off + n) on stream st (a grid shape's range in the shape pipeline)
struct BeadRange {
  cudaStream_t st;
  int off, n;
};
inline BeadRange all_beads(tild_ctx* c) { return {c->stream, 0, c->n_cta_bead}; }

// CH: some system of the engine has charges (the kernels without it carry no charge code)
template <int D, int P, bool CH>
void launch_spread_k(tild_ctx* c, BeadRange r) {
  if (P <= 1 || c->spread_mode == TILD_SPREAD_DIRECT) {
    k_spread_direct<D, P, CH><<<r.n, kTile, 0, r.st>>>(c->pos[c->cur], c->charge, c->cta_bead, c->d_sys, c->rho_fx,
                                                        c->d_status, r.off);
  } else if constexpr (P >= 2) {
    static std::atomic<unsigned long long> attr_devices{0};  // one bit per device with the attribute set
    const unsigned long long bit = 1ull << (c->device & 63);
    if (!(attr_devices.load() & bit)) {
      cudaFuncSetAttribute(k_spread_tiled<D, P, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(sizeof(int) * 12288));
      attr_devices.fetch_or(bit);
    }
    const size_t smem = sizeof(int) * (size_t)c->spread_cap;
    k_spread_tiled<D, P, CH><<<r.n, kTile, smem, r.st>>>(c->pos[c->cur], c->charge, c->cta_bead, c->d_sys, c->rho_fx,
                                                          c->spread_cap, c->d_status, r.off);
  }
}

template <int D, int P>
void launch_spread(tild_ctx* c, BeadRange r) {
  if (r.n == 0) return;
  if (c->any_charges) launch_spread_k<D, P, true>(c, r);
  else launch_spread_k<D, P, false>(c, r);
}

template <int D, int P, bool I, bool X, bool CH>
void launch_gather_k(tild_ctx* c, float* f_out, int f_sys, BeadRange r) {
  if (P >= 2 && c->gather_mode == TILD_GATHER_BOX && c->field_layout == TILD_FIELD_LINEAR) {
    static std::atomic<unsigned long long> attr_devices{0};  // one bit per device with the attribute set
    const unsigned long long bit = 1ull << (c->device & 63);
    if (!(attr_devices.load() & bit)) {
      cudaFuncSetAttribute(k_gather_box<D, P, I, X, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(sizeof(float4) * kGatherBoxMax));
      attr_devices.fetch_or(bit);
    }
    k_gather_box<D, P, I, X, CH><<<r.n, kTile, sizeof(float4) * (size_t)c->gather_cap, r.st>>>(
        c->pos[c->cur], c->pos[c->cur ^ 1], c->noise, c->bead_id, c->bond_nbr, c->bond_info, c->charge, c->g4,
        c->cta_bead, c->d_sys, f_out, f_sys, c->xorwow, c->gather_cap, c->d_status, r.off);
    return;
  }
  if constexpr (I) {
    if (tild_spreads_ahead(c, true)) {
      if constexpr (P >= 2) {
        if (c->spread_mode == TILD_SPREAD_TILED) {  // spread ahead through the shared box
          static std::atomic<unsigned long long> attr_devices{0};  // one bit per device with the attribute set
          const unsigned long long bit = 1ull << (c->device & 63);
          if (!(attr_devices.load() & bit)) {
            cudaFuncSetAttribute(k_gather<D, P, I, X, CH, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(int) * 12288));
            attr_devices.fetch_or(bit);
          }
          k_gather<D, P, I, X, CH, 1><<<r.n, kTile, sizeof(int) * (size_t)c->spread_cap, r.st>>>(
              c->pos[c->cur], c->pos[c->cur ^ 1], c->noise, c->bead_id, c->bond_nbr, c->bond_info, c->charge, c->g4,
              c->cta_bead, c->d_sys, f_out, f_sys, c->xorwow, c->field_layout, c->rho_fx, c->spread_cap,
              c->d_status, r.off);
          return;
        }
      }
      if constexpr (!(D == 3 && P == 3)) {  // no shared memory: all of it as L1
        static std::atomic<unsigned long long> attr_devices2{0};
        const unsigned long long bit = 1ull << (c->device & 63);
        if (!(attr_devices2.load() & bit)) {
          cudaFuncSetAttribute(k_gather<D, P, I, X, CH, 2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxL1);
          attr_devices2.fetch_or(bit);
        }
      }
      k_gather<D, P, I, X, CH, 2><<<r.n, kTile, 0, r.st>>>(  // spread ahead by global atomics
          c->pos[c->cur], c->pos[c->cur ^ 1], c->noise, c->bead_id, c->bond_nbr, c->bond_info, c->charge, c->g4,
          c->cta_bead, c->d_sys, f_out, f_sys, c->xorwow, c->field_layout, c->rho_fx, 0, c->d_status, r.off);
      return;
    }
  }
  if constexpr (!(D == 3 && P == 3)) {
    // no shared memory: all of it as L1 for the force field
    static std::atomic<unsigned long long> attr_devices{0};  // one bit per device with the attribute set
    const unsigned long long bit = 1ull << (c->device & 63);
    if (!(attr_devices.load() & bit)) {
      cudaFuncSetAttribute(k_gather<D, P, I, X, CH, 0>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           cudaSharedmemCarveoutMaxL1);
      attr_devices.fetch_or(bit);
    }
  }
  if constexpr (D == 3 && P == 3) {
    // 4 CTAs of the quarter-warp stencil need 100 KB of shared memory (24 KB of staged stencil
    // records and 1 KB reserved each).  A hint of 40 % of the 228 KB makes the driver take the
    // smallest split that still holds the 4 CTAs, 100 KB, so the rest of the SM's 256 KB is L1 for
    // the force field; without it the 132 KB split is taken (blend gather 0.267 -> 0.253 ms)
    static std::atomic<unsigned long long> attr_devices{0};  // one bit per device with the attribute set
    const unsigned long long bit = 1ull << (c->device & 63);
    if (!(attr_devices.load() & bit)) {
      cudaFuncSetAttribute(k_gather<D, P, I, X, CH, 0>, cudaFuncAttributePreferredSharedMemoryCarveout, 40);
      attr_devices.fetch_or(bit);
    }
  }
  k_gather<D, P, I, X, CH, 0><<<r.n, kTile, 0, r.st>>>(
      c->pos[c->cur], c->pos[c->cur ^ 1], c->noise, c->bead_id, c->bond_nbr, c->bond_info, c->charge, c->g4,
      c->cta_bead, c->d_sys, f_out, f_sys, c->xorwow, c->field_layout, nullptr, 0, c->d_status, r.off);
}

template <int D, int P, bool I, bool X>
void launch_gather_ch(tild_ctx* c, float* f_out, int f_sys, BeadRange r) {
  if (r.n == 0) return;
  if (c->any_charges) launch_gather_k<D, P, I, X, true>(c, f_out, f_sys, r);
  else launch_gather_k<D, P, I, X, false>(c, f_out, f_sys, r);
}

template <int D, int P>
void launch_gather(tild_ctx* c, bool integ, float* f_out, int f_sys, BeadRange r) {
  const bool xw = c->rng == TILD_RNG_XORWOW;
  if (integ) {
    if (xw) launch_gather_ch<D, P, true, true>(c, f_out, f_sys, r);
    else launch_gather_ch<D, P, true, false>(c, f_out, f_sys, r);
  } else {
    launch_gather_ch<D, P, false, false>(c, f_out, f_sys, r);
  }
}

template <int D>
void dispatch_p_spread(tild_ctx* c, BeadRange r) {
  switch (c->P) {
    case 0: launch_spread<D, 0>(c, r); break;
    case 1: launch_spread<D, 1>(c, r); break;
    case 2: launch_spread<D, 2>(c, r); break;
    case 3: launch_spread<D, 3>(c, r); break;
    default: launch_spread<D, 4>(c, r); break;
  }
}

template <int D>
void dispatch_p_gather(tild_ctx* c, bool integ, float* f_out, int f_sys, BeadRange r) {
  switch (c->P) {
    case 0: launch_gather<D, 0>(c, integ, f_out, f_sys, r); break;
    case 1: launch_gather<D, 1>(c, integ, f_out, f_sys, r); break;
    case 2: launch_gather<D, 2>(c, integ, f_out, f_sys, r); break;
    case 3: launch_gather<D, 3>(c, integ, f_out, f_sys, r); break;
    default: launch_gather<D, 4>(c, integ, f_out, f_sys, r); break;
  }
}

// interleave over grid blocks [off, off + n) on stream st
void launch_interleave(tild_ctx* c, cudaStream_t st, int off, int n) {
  if (n == 0) return;
  int* blk0 = c->cta_grid + c->n_cta_grid;
  if (c->D == 3)
    k_interleave<3><<<n, 256, 0, st>>>(c->gfield, reinterpret_cast<const float2*>(c->gk), c->g4, c->cta_grid, blk0,
                                       c->d_sys, c->field_layout, off);
  else
    k_interleave<2><<<n, 256, 0, st>>>(c->gfield, reinterpret_cast<const float2*>(c->gk), c->g4, c->cta_grid, blk0,
                                       c->d_sys, c->field_layout, off);
}

// k-space multiply over spectrum blocks [off, off + n) (all of them by default) on stream st
template <int D>
void launch_kmul(tild_ctx* c, bool integ, cudaStream_t st = nullptr, int off = 0, int n = -1) {
  const float2* rk = reinterpret_cast<const float2*>(c->rhok);
  float2* gk = reinterpret_cast<float2*>(c->gk);
  int* blk0 = c->cta_spec + c->n_cta_spec;  // first-block table stored after the lookup table
  if (n < 0) n = c->n_cta_spec;
  if (!st) st = c->stream;
  if (n == 0) return;
  switch (c->maxT) {
    case 1: k_kmul<D, 1><<<n, 256, 0, st>>>(rk, gk, c->utab, c->ctab, c->kd, c->cta_spec, blk0, c->d_sys, integ, off); break;
    case 2: k_kmul<D, 2><<<n, 256, 0, st>>>(rk, gk, c->utab, c->ctab, c->kd, c->cta_spec, blk0, c->d_sys, integ, off); break;
    case 3: k_kmul<D, 3><<<n, 256, 0, st>>>(rk, gk, c->utab, c->ctab, c->kd, c->cta_spec, blk0, c->d_sys, integ, off); break;
    case 4: k_kmul<D, 4><<<n, 256, 0, st>>>(rk, gk, c->utab, c->ctab, c->kd, c->cta_spec, blk0, c->d_sys, integ, off); break;
    default: k_kmul<D, 0><<<n, 256, 0, st>>>(rk, gk, c->utab, c->ctab, c->kd, c->cta_spec, blk0, c->d_sys, integ, off); break;
  }
}

// fork the auxiliary streams off the main stream, and join them back
int fork(tild_ctx* c) {
  if (c->lanes == 0) return 0;
  if (tild_check(c, cudaEventRecord(c->ev_fork, c->stream), "fork")) return 1;
  for (int k = 0; k < c->lanes; k++)
    if (tild_check(c, cudaStreamWaitEvent(c->aux[k], c->ev_fork, 0), "fork wait")) return 1;
  return 0;
}

// the bucket's fixed-point densities to FP32 (clearing the accumulator): planar channels, or
// complex channel pairs when its forward transform is paired
void launch_fix(tild_ctx* c, const Bucket& b, cudaStream_t st) {
  const long long M = (long long)b.nx[0] * b.nx[1] * b.nx[2];
  if (b.fwd_packed) {
    const long long np = b.channels / 2;
    k_fix_to_pairs<<<nblk(np * M, 256), 256, 0, st>>>(c->rho_fx + b.grid0, reinterpret_cast<float2*>(c->rho + b.grid0),
                                                      np, M);
  } else {
    k_fix_to_float<<<nblk((long long)b.channels * M, 256), 256, 0, st>>>(c->rho_fx + b.grid0, c->rho + b.grid0,
                                                                         (long long)b.channels * M);
  }
  c->launches++;
}

// the bucket's batched forward transform: R2C per channel, or C2C per channel pair (out of place,
// the pair spectra into rhok; the paired real-space densities stay for density reads)
int exec_forward(tild_ctx* c, const Bucket& b) {
  if (b.fwd_packed)
    return tild_check_fft(c, cufftExecC2C(b.c2c_fwd, reinterpret_cast<cufftComplex*>(c->rho + b.grid0),
                                          c->rhok + b.spec0, CUFFT_FORWARD), "C2C forward");
  return tild_check_fft(c, cufftExecR2C(b.r2c, c->rho + b.grid0, c->rhok + b.spec0), "R2C");
}

// the bucket's batched inverse transform: C2R per channel and direction, or C2C per channel pair
int exec_inverse(tild_ctx* c, const Bucket& b) {
  if (b.packed)
    return tild_check_fft(c, cufftExecC2C(b.c2c, c->gk + b.spec0 * c->D, c->gk + b.spec0 * c->D, CUFFT_INVERSE),
                          "C2C");  // in place: the interleave reads the pair fields from gk
  return tild_check_fft(c, cufftExecC2R(b.c2r, c->gk + b.spec0 * c->D, c->gfield + b.grid0 * c->D), "C2R");
}

int join(tild_ctx* c) {
  for (int k = 0; k < c->lanes; k++) {
    if (tild_check(c, cudaEventRecord(c->ev_join[k], c->aux[k]), "join")) return 1;
    if (tild_check(c, cudaStreamWaitEvent(c->stream, c->ev_join[k], 0), "join wait")) return 1;
  }
  return 0;
}

}  // namespace

int tild_run_forces(tild_ctx* c, bool integrate, float* f_bead, int f_sys) {
  if (integrate && c->sort_interval > 0 && c->steps_since_sort >= c->sort_interval) {
    tild_mark(c, STAGE_SORT);
    int rs = tild_sort_beads(c);
    if (rs) return rs;
  }
  const std::vector<char> on = integrate ? tild_buckets_on(c) : std::vector<char>(c->buckets.size(), 1);
  if (c->fft_pipeline >= 2 && c->lanes > 0 && c->fields.empty()) {
    // each grid shape runs its whole step in order on its stream: spread, conversion, R2C,
    // k-space multiply, C2R, interleave and gather, so one shape's transforms overlap another's
    // particle kernels (one profiling stage).  Idle shapes still spread and gather, which keeps
    // their densities current and their positions held.
    tild_mark(c, STAGE_R2C);
    if (fork(c)) return TILD_ERR_CUDA;
    for (size_t bi = 0; bi < c->buckets.size(); bi++) {
      const Bucket& b = c->buckets[bi];
      cudaStream_t bs = b.lane >= 0 ? c->aux[b.lane] : c->stream;
      const BeadRange r{bs, b.cta_bead0, b.n_cta_bead};
      if (!c->rho_ahead) {
        if (c->D == 3) dispatch_p_spread<3>(c, r);
        else dispatch_p_spread<2>(c, r);
        c->launches++;
      }
      launch_fix(c, b, bs);
      if (on[bi]) {
        if (exec_forward(c, b)) return TILD_ERR_CUDA;
        if (c->D == 3) launch_kmul<3>(c, integrate, bs, b.cta_spec0, b.n_cta_spec);
        else launch_kmul<2>(c, integrate, bs, b.cta_spec0, b.n_cta_spec);
        if (exec_inverse(c, b))
          return TILD_ERR_CUDA;
        launch_interleave(c, bs, b.cta_grid0, b.n_cta_grid);
        c->launches += 2;
      }
      if (c->D == 3) dispatch_p_gather<3>(c, integrate, f_bead, f_sys, r);
      else dispatch_p_gather<2>(c, integrate, f_bead, f_sys, r);
      c->launches++;
    }
    if (join(c)) return TILD_ERR_CUDA;
    if (tild_check(c, cudaGetLastError(), "shape pipeline")) return TILD_ERR_CUDA;
    c->rho_ahead = false;  // the conversions cleared the accumulator
    return tild_finish_forces(c, integrate, f_bead, f_sys, true, true);
  }
  tild_mark(c, STAGE_SPREAD);
  if (!c->rho_ahead) {  // else the previous step's gather spread these positions already
    if (c->D == 3) dispatch_p_spread<3>(c, all_beads(c));
    else dispatch_p_spread<2>(c, all_beads(c));
    c->launches++;
  }
  c->rho_ahead = false;  // the conversion below clears the accumulator
  if (c->fft_pipeline >= 1 && c->lanes > 0) {
    // each grid shape runs conversion, R2C, k-space multiply and C2R in order on its stream, so
    // one shape's transforms overlap another's element-wise passes (one profiling stage)
    tild_mark(c, STAGE_R2C);
    if (fork(c)) return TILD_ERR_CUDA;
    for (size_t bi = 0; bi < c->buckets.size(); bi++) {
      const Bucket& b = c->buckets[bi];
      cudaStream_t bs = b.lane >= 0 ? c->aux[b.lane] : c->stream;
      launch_fix(c, b, bs);
      if (!on[bi]) continue;
      if (exec_forward(c, b)) return TILD_ERR_CUDA;
      if (c->D == 3) launch_kmul<3>(c, integrate, bs, b.cta_spec0, b.n_cta_spec);
      else launch_kmul<2>(c, integrate, bs, b.cta_spec0, b.n_cta_spec);
      c->launches++;
      if (exec_inverse(c, b))
        return TILD_ERR_CUDA;
      if (c->fields.empty()) {  // fieldphase edits the planar fields first when present
        launch_interleave(c, bs, b.cta_grid0, b.n_cta_grid);
        c->launches++;
      }
    }
    if (join(c)) return TILD_ERR_CUDA;
    if (tild_check(c, cudaGetLastError(), "shape pipeline")) return TILD_ERR_CUDA;
    return tild_finish_forces(c, integrate, f_bead, f_sys, c->fields.empty(), false);
  }
  tild_mark(c, STAGE_ZERO);
  bool any_fwd_packed = false;
  for (const Bucket& b : c->buckets) any_fwd_packed = any_fwd_packed || b.fwd_packed;
  if (any_fwd_packed) {  // paired shapes convert into their own layout
    for (const Bucket& b : c->buckets) launch_fix(c, b, c->stream);
  } else {
    k_fix_to_float<<<nblk(c->grid_total, 256), 256, 0, c->stream>>>(c->rho_fx, c->rho, c->grid_total);
    c->launches++;
  }
  if (tild_check(c, cudaGetLastError(), "spread")) return TILD_ERR_CUDA;
  tild_mark(c, STAGE_R2C);
  if (fork(c)) return TILD_ERR_CUDA;
  for (size_t bi = 0; bi < c->buckets.size(); bi++) {
    const Bucket& b = c->buckets[bi];
    if (on[bi] && exec_forward(c, b)) return TILD_ERR_CUDA;
  }
  if (join(c)) return TILD_ERR_CUDA;
  tild_mark(c, STAGE_KMUL);
  if (c->D == 3) launch_kmul<3>(c, integrate);
  else launch_kmul<2>(c, integrate);
  c->launches++;
  if (tild_check(c, cudaGetLastError(), "kmul")) return TILD_ERR_CUDA;
  tild_mark(c, STAGE_C2R);
  if (fork(c)) return TILD_ERR_CUDA;
  for (size_t bi = 0; bi < c->buckets.size(); bi++) {
    const Bucket& b = c->buckets[bi];
    if (on[bi] && exec_inverse(c, b))
      return TILD_ERR_CUDA;
  }
  if (join(c)) return TILD_ERR_CUDA;
  return tild_finish_forces(c, integrate, f_bead, f_sys, false, false);
}

// fieldphase, interleave (unless the shape pipeline did it), gather (+ bonds + integrators) and
// the step tail
int tild_finish_forces(tild_ctx* c, bool integrate, float* f_bead, int f_sys, bool interleaved, bool gathered) {
  if (!c->fields.empty()) tild_mark(c, STAGE_FIELD);
  for (const FieldK& fk : c->fields) {
    const SysHost& h = c->sys[fk.sys];
    k_fieldphase_apply<<<nblk(h.g.M, 256), 256, 0, c->stream>>>(c->gfield + h.grid0 * c->D, c->rho + h.grid0,
                                                                 c->frfield + fk.fr0, fk.a, fk.b, c->D, h.g.M);
    c->launches++;
  }
  if (!interleaved) {
    tild_mark(c, STAGE_INTERLEAVE);
    launch_interleave(c, c->stream, 0, c->n_cta_grid);
    c->launches++;
  }
  if (!gathered) {
    tild_mark(c, STAGE_GATHER);
    if (c->D == 3) dispatch_p_gather<3>(c, integrate, f_bead, f_sys, all_beads(c));
    else dispatch_p_gather<2>(c, integrate, f_bead, f_sys, all_beads(c));
    c->launches++;
    if (tild_check(c, cudaGetLastError(), "gather")) return TILD_ERR_CUDA;
  }
  c->rho_ahead = tild_spreads_ahead(c, integrate);
  if (integrate) {
    tild_mark(c, STAGE_TAIL);
    k_advance_steps<<<nblk(c->nsys, 128), 128, 0, c->stream>>>(c->d_sys, c->nsys);
    c->launches++;
    c->cur ^= 1;
    c->steps_since_sort++;
  }
  for (int s = 0; s < c->nsys; s++) {
    SysHost& h = c->sys[s];
    if (!h.active) continue;
    if (integrate) {
      h.step++;
      c->h_sys[s].step = h.step;
    }
    h.forces_step = h.step;
    h.have_forces = true;
  }
  return TILD_OK;
}

// A system's densities as planar FP32 channels [(T + C)][M] into dst (device memory) on stream st:
// a copy, or the de-interleave of its paired layout.
int tild_density_planar(tild_ctx* c, int s, float* dst, cudaStream_t st) {
  const SysHost& h = c->sys[s];
  const long long M = h.g.M;
  if (c->h_sys[s].fwd_packed) {
    const long long np = (h.T + h.C) / 2;
    k_pairs_to_planar<<<nblk(np * M, 256), 256, 0, st>>>(reinterpret_cast<const float2*>(c->rho + h.grid0), dst, np, M);
    c->launches++;
    return tild_check(c, cudaGetLastError(), "densities to planar") ? TILD_ERR_CUDA : TILD_OK;
  }
  return tild_check(c, cudaMemcpyAsync(dst, c->rho + h.grid0, sizeof(float) * (size_t)(h.T + h.C) * M,
                                       cudaMemcpyDeviceToDevice, st), "copy densities") ? TILD_ERR_CUDA : TILD_OK;
}

// A system's density half spectra in the R2C layout [(T + C)][Mh], valid after its last force
// evaluation: rhok itself, or (paired forward transform) unpacked into the force spectra buffer,
// which holds nothing between steps.
const float2* tild_half_spectra(tild_ctx* c, int s) {
  const SysHost& h = c->sys[s];
  const SysDev& d = c->h_sys[s];
  if (!d.fwd_packed) return reinterpret_cast<const float2*>(c->rhok) + h.spec0;
  float2* half = reinterpret_cast<float2*>(c->gk) + h.spec0;
  k_unpack_half<<<nblk(h.g.Mh, 256), 256, 0, c->stream>>>(reinterpret_cast<const float2*>(c->rhok) + d.rkp0, half,
                                                           (h.T + h.C) / 2, h.g, h.D);
  c->launches++;
  return half;
}
