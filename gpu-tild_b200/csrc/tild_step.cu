// tild_step.cu — the per-step hot path: spread -> batched R2C -> k-space multiply -> batched C2R
// -> fused gather + bonds + integrators.
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
#include "tild_internal.cuh"
#include <climits>

namespace {

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// ---------------------------------------------------------------------------------------------
// Spreading: d_charge_grid / d_charge_grid_charges (device_grid_utils.cu:111-343)
// ---------------------------------------------------------------------------------------------
// Tiled spreading for slot-sorted beads.  One CTA takes 256 consecutive slots; their stencil
// nodes are accumulated into a shared-memory box (relative to the first bead, periodic offsets
// folded into [-N/2, N/2]) and the box is added to the global grid once.  Accumulation is in
// 64-bit fixed point (weight * 2^32, native integer atomics): integer sums do not depend on the
// order of the additions, so the densities are bitwise reproducible whatever the slot order or
// the scheduling, and carry ~1e-10 absolute error before the single FP32 rounding.  When the box
// does not fit (unsorted or widely spread chunks) the CTA adds each node to the global
// fixed-point grid directly.
__device__ __forceinline__ int fold_rel(int r, int N) {
  r %= N;
  if (r < 0) r += N;
  if (r > N / 2) r -= N;
  return r;
}

__device__ __forceinline__ int pmod(int n, int N) {
  n %= N;
  return n < 0 ? n + N : n;
}

constexpr double kFix = 4294967296.0;           // 2^32
constexpr int kMaxRows = 1024;                  // (y, z) rows of a shared-memory spread box
constexpr double kInvFix = 1.0 / 4294967296.0;

__device__ __forceinline__ unsigned long long to_fix(float v) {
  return (unsigned long long)__double2ll_rn((double)v * kFix);
}

// Chunk bounding box of the beads' stencil bases, relative to the chunk's first bead.
// Returns false when no bead of the chunk is finite.  Every thread of the block must call it.
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
    float Wd[P + 1];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      s_g0[d] = (d < D && isfinite(x0[d])) ? axis_base<P>(x0[d], g.dx[d], Wd) : 0;
      s_min[d] = INT_MAX;
      s_max[d] = INT_MIN;
    }
  }
  __syncthreads();
}

template <int D, int P>
__global__ void __launch_bounds__(256) k_spread_tiled(const float4* __restrict__ pos, const float* __restrict__ charge,
                                                     int ns, Geom g, unsigned long long* __restrict__ rho_fx, int T,
                                                     int C, int cap, int kbits, int* status) {
  // shared box: 32-bit fixed point with 2^kbits per unit (native integer shared atomics); kbits is
  // chosen per context so that 256 beads at the largest weight cannot overflow
  extern __shared__ int smi[];
  __shared__ int s_g0[3], s_min[3], s_max[3];
  __shared__ long long s_row[kMaxRows];
  const int i0 = blockIdx.x * blockDim.x;
  const int i = i0 + threadIdx.x;
  chunk_origin<D, P>(pos, i0, g, s_g0, s_min, s_max);
  float W[3][P + 1];
  int rel[3] = {0, 0, 0};
  int t = 0;
  float q = 0.f;
  bool ok = false;
  if (i < ns) {
    const float4 p = pos[i];
    const float xs[3] = {p.x, p.y, p.z};
    ok = isfinite(p.x) && isfinite(p.y) && (D == 2 || isfinite(p.z));
    if (!ok) {
      atomicOr(status, ST_NONFINITE_POS);
    } else {
      t = tild_type_of(p.w);
      q = C ? charge[i] : 0.f;
#pragma unroll
      for (int d = 0; d < D; d++) rel[d] = fold_rel(axis_base<P>(xs[d], g.dx[d], W[d]) - s_g0[d], g.nx[d]);
    }
  }
  int mn[3], ext[3];
  long long vol;
  if (!chunk_box<D, P>(ok, rel, s_min, s_max, mn, ext, vol)) return;
  const int nch = T + C;
  const long long M = g.M;
  const float ig = 1.0f / g.gvol;
  const bool qc = C && q != 0.f;
  if (vol * nch <= cap && ext[0] <= 64 && ext[1] * ext[2] <= kMaxRows) {
    const int tot = (int)vol * nch;
    for (int k = threadIdx.x; k < tot; k += blockDim.x) smi[k] = 0;
    __syncthreads();
    if (ok) {
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
    // flush: one warp per box row (y, z) and channel, lanes along x; exact shift to the 2^32 grid
    const int rows_per = ext[1] * ext[2];
    for (int yz = threadIdx.x; yz < rows_per; yz += blockDim.x) {
      const int ly = yz % ext[1], lz = yz / ext[1];
      s_row[yz] = (long long)g.nx[0] * (pmod(s_g0[1] + mn[1] + ly, g.nx[1]) +
                                        (long long)g.nx[1] * (D == 3 ? pmod(s_g0[2] + mn[2] + lz, g.nx[2]) : 0));
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int bx = pmod(s_g0[0] + mn[0], g.nx[0]);
    int xoff[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
      int xg = bx + lane + 32 * k;
      while (xg >= g.nx[0]) xg -= g.nx[0];
      xoff[k] = xg;
    }
    const int sh = 32 - kbits;
    for (int ch = 0; ch < nch; ch++) {
      const int* sch = smi + (long long)ch * vol;
      unsigned long long* gch = rho_fx + ch * M;
      for (int yz = warp; yz < rows_per; yz += nwarps) {
        const int* srow = sch + (long long)yz * ext[0];
        unsigned long long* grow = gch + s_row[yz];
#pragma unroll
        for (int k = 0; k < 2; k++) {
          const int lx = lane + 32 * k;
          if (lx < ext[0]) {
            const int v = srow[lx];
            if (v != 0) atomicAdd(grow + xoff[k], (unsigned long long)((long long)v << sh));
          }
        }
      }
    }
  } else if (ok) {
    int idx[3][P + 1];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int a = 0; a <= P; a++) idx[d][a] = pmod(s_g0[d] + rel[d] + a, g.nx[d]);
    unsigned long long* rt = rho_fx + (long long)t * M;
    unsigned long long* rc = rho_fx + (long long)T * M;
#pragma unroll
    for (int ix = 0; ix <= P; ix++)
#pragma unroll
      for (int iy = 0; iy <= P; iy++) {
        const long long row = idx[0][ix] + (long long)idx[1][iy] * g.nx[0];
        const float wxy = W[0][ix] * W[1][iy] * ig;
        if (D == 3) {
#pragma unroll
          for (int iz = 0; iz <= P; iz++) {
            const long long m = row + (long long)idx[2][iz] * g.nx[1] * g.nx[0];
            const float W3 = wxy * W[2][iz];
            atomicAdd(rt + m, to_fix(W3));
            if (qc) atomicAdd(rc + m, to_fix(W3 * q));
          }
        } else {
          atomicAdd(rt + row, to_fix(wxy));
          if (qc) atomicAdd(rc + row, to_fix(wxy * q));
        }
      }
  }
}

// fixed-point grid -> FP32 density, clearing the accumulator for the next step
__global__ void k_fix_to_float(unsigned long long* __restrict__ fx, float* __restrict__ rho, long long n) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const long long v = (long long)fx[k];
  rho[k] = (float)((double)v * kInvFix);
  fx[k] = 0ull;
}

// ---------------------------------------------------------------------------------------------
// k-space multiply (replaces d_prepareForceKSpace, device_array_utils.cu:298-312, for every
// style and side, and d_prepareElectrostaticPotential / d_prepareElectricField :199-241)
// ---------------------------------------------------------------------------------------------
struct KArgs {
  int nstyle;
  int a[TILD_MAX_STYLES];
  int b[TILD_MAX_STYLES];
  float scale[TILD_MAX_STYLES];
};

template <int D, int NT>
__global__ void __launch_bounds__(256) k_kmul(const float2* __restrict__ rhok, float2* __restrict__ gk,
                                             const float* __restrict__ utab, const float* __restrict__ ctab,
                                             const float* __restrict__ kd, Geom g, int T, int C, KArgs ka) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= g.Mh) return;
  const int ix = (int)(h % g.nxh);
  const long long r = h / g.nxh;
  const int iy = (int)(r % g.nx[1]);
  const int iz = (int)(r / g.nx[1]);
  float kv[3];
  kv[0] = kd[ix];
  kv[1] = kd[g.nx[0] + iy];
  kv[2] = (D == 3) ? kd[g.nx[0] + g.nx[1] + iz] : 0.f;
  const long long Mh = g.Mh;
  float2 rk[NT], phi[NT];
#pragma unroll
  for (int t = 0; t < NT; t++) {
    rk[t] = (t < T) ? rhok[(long long)t * Mh + h] : make_float2(0.f, 0.f);
    phi[t] = make_float2(0.f, 0.f);
  }
  for (int s = 0; s < ka.nstyle; s++) {
    const float u = utab[(long long)s * Mh + h] * ka.scale[s];
    const int a = ka.a[s], b = ka.b[s];
    // explicit selects keep rk[] and phi[] in registers
    float2 ra = make_float2(0.f, 0.f), rb = make_float2(0.f, 0.f);
#pragma unroll
    for (int t = 0; t < NT; t++) {
      if (t == a) ra = rk[t];
      if (t == b) rb = rk[t];
    }
#pragma unroll
    for (int t = 0; t < NT; t++) {
      if (t == a) { phi[t].x += u * rb.x; phi[t].y += u * rb.y; }
      if (t == b) { phi[t].x += u * ra.x; phi[t].y += u * ra.y; }
    }
  }
#pragma unroll
  for (int t = 0; t < NT; t++) {
    if (t >= T) break;
#pragma unroll
    for (int d = 0; d < D; d++)  // -i k_d Phi
      gk[((long long)t * D + d) * Mh + h] = make_float2(kv[d] * phi[t].y, -kv[d] * phi[t].x);
  }
  if (C) {
    const float2 rc = rhok[(long long)T * Mh + h];
    const float cm = ctab[h];
    const float2 pc = make_float2(cm * rc.x, cm * rc.y);
#pragma unroll
    for (int d = 0; d < D; d++) gk[((long long)T * D + d) * Mh + h] = make_float2(kv[d] * pc.y, -kv[d] * pc.x);
  }
}

// Generic channel count (T > TILD_MAXT_FAST): same arithmetic with local arrays.
template <int D>
__global__ void k_kmul_generic(const float2* __restrict__ rhok, float2* __restrict__ gk, const float* __restrict__ utab,
                               const float* __restrict__ ctab, const float* __restrict__ kd, Geom g, int T, int C,
                               KArgs ka) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= g.Mh) return;
  const int ix = (int)(h % g.nxh);
  const long long r = h / g.nxh;
  const int iy = (int)(r % g.nx[1]);
  const int iz = (int)(r / g.nx[1]);
  float kv[3] = {kd[ix], kd[g.nx[0] + iy], (D == 3) ? kd[g.nx[0] + g.nx[1] + iz] : 0.f};
  const long long Mh = g.Mh;
  float2 phi[TILD_MAX_TYPES];
  for (int t = 0; t < T; t++) phi[t] = make_float2(0.f, 0.f);
  for (int s = 0; s < ka.nstyle; s++) {
    const float u = utab[(long long)s * Mh + h] * ka.scale[s];
    const int a = ka.a[s], b = ka.b[s];
    const float2 ra = rhok[(long long)a * Mh + h], rb = rhok[(long long)b * Mh + h];
    phi[a].x += u * rb.x; phi[a].y += u * rb.y;
    phi[b].x += u * ra.x; phi[b].y += u * ra.y;
  }
  for (int t = 0; t < T; t++)
    for (int d = 0; d < D; d++) gk[((long long)t * D + d) * Mh + h] = make_float2(kv[d] * phi[t].y, -kv[d] * phi[t].x);
  if (C) {
    const float2 rc = rhok[(long long)T * Mh + h];
    const float cm = ctab[h];
    for (int d = 0; d < D; d++)
      gk[((long long)T * D + d) * Mh + h] = make_float2(kv[d] * cm * rc.y, -kv[d] * cm * rc.x);
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

// ---------------------------------------------------------------------------------------------
// Gather + bonds + integrators (d_add_grid_forces{2D,3D}, d_add_grid_forces_charges_*,
// device_grid_utils.cu:346-452; d_bonds, device_bonds.cu:4-60; d_GJF_integrator,
// device_GJF_integrator.cu:4-62; d_EM_integrator, device_EM_integrator.cu:5-36)
// ---------------------------------------------------------------------------------------------
struct GArgs {
  int64_t step;
  uint64_t seed;
  float delt, noise_mag;
  int n_integ;
  int integ_kind[TILD_MAX_INTEGRATORS];
  int type_mask[TILD_MAX_TYPES];
  float mass[TILD_MAX_TYPES];
  float diff[TILD_MAX_TYPES];
  float bond_k[TILD_MAX_BOND_TYPES];
  float bond_req[TILD_MAX_BOND_TYPES];
};

// Interleave the C2R output [(T+C)][D][M] into one float4 (-dPhi/dx, -dPhi/dy, -dPhi/dz, 0) per
// grid point and channel, so the gather reads a stencil node with a single 16-byte load.
__global__ void k_interleave(const float* __restrict__ planar, float4* __restrict__ g4, int nch, int D, long long M) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= M) return;
  for (int ch = 0; ch < nch; ch++) {
    const float* src = planar + (long long)ch * D * M + m;
    g4[(long long)ch * M + m] = make_float4(src[0], src[M], D == 3 ? src[2 * M] : 0.f, 0.f);
  }
}

template <int D, int P>
__device__ __forceinline__ void gather4(const float4* __restrict__ F, const float (&W)[3][P + 1],
                                        const int (&idx)[3][P + 1], const Geom& g, float (&acc)[3]) {
#pragma unroll
  for (int ix = 0; ix <= P; ix++)
#pragma unroll
    for (int iy = 0; iy <= P; iy++) {
      const float wxy = W[0][ix] * W[1][iy];
      const long long row = idx[0][ix] + (long long)idx[1][iy] * g.nx[0];
      if (D == 3) {
#pragma unroll
        for (int iz = 0; iz <= P; iz++) {
          const float4 v = __ldg(F + row + (long long)idx[2][iz] * g.nx[1] * g.nx[0]);
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

template <int D, int P, bool INTEG, bool XW>
__global__ void __launch_bounds__(256, (P >= 4 ? 2 : 3)) k_gather(const float4* __restrict__ pos_in, float4* __restrict__ pos_io,
                                                  float* __restrict__ noise, const int* __restrict__ bead_id,
                                                  const int* __restrict__ bond_nbr, const int* __restrict__ bond_info,
                                                  const float* __restrict__ charge, const float4* __restrict__ g4,
                                                  Geom g, int T, int C, GArgs ga, float* __restrict__ f_out,
                                                  curandStateXORWOW_t* __restrict__ xw, int ns, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const float4 p = pos_in[i];
  float x[3] = {p.x, p.y, p.z};
  if (!(isfinite(p.x) && isfinite(p.y) && (D == 2 || isfinite(p.z)))) {
    atomicOr(status, ST_NONFINITE_POS);
    return;  // left in place; the host reports TILD_ERR_NAN
  }
  const int t = tild_type_of(p.w);
  const long long M = g.M;
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
    if (C) {
      const float q = charge[i];
      if (q != 0.f) {
        float e[3] = {0.f, 0.f, 0.f};
        gather4<D, P>(g4 + (long long)T * M, W, idx, g, e);
#pragma unroll
        for (int d = 0; d < D; d++) f[d] += e[d] * q;
      }
    }
    gather4<D, P>(g4 + (long long)t * M, W, idx, g, f);
  }
  // bonds
  const int info = bond_info[i];
  const int nb = info & 3;
  for (int bb = 0; bb < nb; bb++) {
    const int j = bond_nbr[3 * i + bb];
    const int bt = (info >> (8 + 8 * bb)) & 0xff;
    const float4 pj = pos_in[j];
    const float xj[3] = {pj.x, pj.y, pj.z};
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
      mf = 2.0f * ga.bond_k[bt] * (mdr - ga.bond_req[bt]) / mdr;
    }
#pragma unroll
    for (int d = 0; d < D; d++) f[d] -= mf * dr[d];
  }
  const int bid = bead_id[i];
  if (f_out) {
#pragma unroll
    for (int d = 0; d < D; d++) f_out[(long long)bid * D + d] = f[d];
  }
  if (!INTEG) return;
  // integrators in input order (integrator.cu:24-39 is called for each in turn)
  const int mask = ga.type_mask[t];
  const float4 po = pos_io[i];  // x_{n-1} (GJF xo)
  float xo[3] = {po.x, po.y, po.z};
  float on[3] = {0.f, 0.f, 0.f};
  bool any_gjf = false;
  curandStateXORWOW_t st;
  if (XW && mask) st = xw[i];
  for (int ig = 0; ig < ga.n_integ; ig++) {
    if (!(mask & (1 << ig))) continue;
    float z[3];
    if (XW) {
#pragma unroll
      for (int d = 0; d < D; d++) z[d] = curand_normal(&st);
    } else {
      philox_normal3(ga.seed, (uint32_t)bid, ga.step, (uint32_t)ig, z);
    }
    if (ga.integ_kind[ig] == TILD_INTEGRATOR_GJF) {
      if (!any_gjf) {
#pragma unroll
        for (int d = 0; d < D; d++) on[d] = noise[3 * (long long)i + d];
        any_gjf = true;
      }
      const float m = ga.mass[t], df = ga.diff[t], delt = ga.delt;
      const float b = m / (m + delt / (2.0f * df));
      const float a = (1.0f - delt / (2.0f * df * m)) / (1.0f + delt / (2.0f * df * m));
      const float delt2 = delt * delt;
#pragma unroll
      for (int d = 0; d < D; d++) {
        const float nn = ga.noise_mag / df * z[d];
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
        float xn = x[d] + ga.delt * f[d] + ga.noise_mag * z[d];
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

template <int D, int P>
void launch_spread(tild_ctx* c) {
  const size_t smem = sizeof(int) * (size_t)c->spread_cap;
  cudaFuncSetAttribute(k_spread_tiled<D, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_spread_tiled<D, P><<<nblk(c->ns, 256), 256, smem, c->stream>>>(c->pos[c->cur], c->charge, c->ns, c->g, c->rho_fx,
                                                                    c->T, c->C, c->spread_cap, c->spread_kbits,
                                                                    c->d_status);
}

template <int D, int P, bool I, bool X>
void launch_gather_k(tild_ctx* c, const GArgs& ga, float* f_out) {
  k_gather<D, P, I, X><<<nblk(c->ns, 256), 256, 0, c->stream>>>(
      c->pos[c->cur], c->pos[c->cur ^ 1], c->noise, c->bead_id, c->bond_nbr, c->bond_info, c->charge, c->g4, c->g,
      c->T, c->C, ga, f_out, c->xorwow, c->ns, c->d_status);
}

template <int D, int P>
void launch_gather(tild_ctx* c, const GArgs& ga, bool integ, float* f_out) {
  const bool xw = c->cfg.rng == TILD_RNG_XORWOW;
  if (integ) {
    if (xw) launch_gather_k<D, P, true, true>(c, ga, f_out);
    else launch_gather_k<D, P, true, false>(c, ga, f_out);
  } else {
    launch_gather_k<D, P, false, false>(c, ga, f_out);
  }
}

template <int D>
void dispatch_p_spread(tild_ctx* c) {
  switch (c->p) {
    case 0: launch_spread<D, 0>(c); break;
    case 1: launch_spread<D, 1>(c); break;
    case 2: launch_spread<D, 2>(c); break;
    case 3: launch_spread<D, 3>(c); break;
    default: launch_spread<D, 4>(c); break;
  }
}

template <int D>
void dispatch_p_gather(tild_ctx* c, const GArgs& ga, bool integ, float* f_out) {
  switch (c->p) {
    case 0: launch_gather<D, 0>(c, ga, integ, f_out); break;
    case 1: launch_gather<D, 1>(c, ga, integ, f_out); break;
    case 2: launch_gather<D, 2>(c, ga, integ, f_out); break;
    case 3: launch_gather<D, 3>(c, ga, integ, f_out); break;
    default: launch_gather<D, 4>(c, ga, integ, f_out); break;
  }
}

template <int D>
void launch_kmul(tild_ctx* c, const KArgs& ka) {
  const unsigned nb = nblk(c->g.Mh, 256);
  const float2* rk = reinterpret_cast<const float2*>(c->rhok);
  float2* gk = reinterpret_cast<float2*>(c->gk);
  switch (c->T) {
    case 1: k_kmul<D, 1><<<nb, 256, 0, c->stream>>>(rk, gk, c->utab, c->ctab, c->kd, c->g, c->T, c->C, ka); break;
    case 2: k_kmul<D, 2><<<nb, 256, 0, c->stream>>>(rk, gk, c->utab, c->ctab, c->kd, c->g, c->T, c->C, ka); break;
    case 3: k_kmul<D, 3><<<nb, 256, 0, c->stream>>>(rk, gk, c->utab, c->ctab, c->kd, c->g, c->T, c->C, ka); break;
    case 4: k_kmul<D, 4><<<nb, 256, 0, c->stream>>>(rk, gk, c->utab, c->ctab, c->kd, c->g, c->T, c->C, ka); break;
    default: k_kmul_generic<D><<<nb, 256, 0, c->stream>>>(rk, gk, c->utab, c->ctab, c->kd, c->g, c->T, c->C, ka); break;
  }
}

}  // namespace

int tild_run_spread(tild_ctx* c) {
  // the fixed-point accumulator is all zeros here: it starts zeroed and k_fix_to_float clears it
  tild_mark(c, STAGE_SPREAD);
  if (c->D == 3) dispatch_p_spread<3>(c);
  else dispatch_p_spread<2>(c);
  c->launches++;
  tild_mark(c, STAGE_ZERO);
  const long long n = (long long)(c->T + c->C) * c->g.M;
  k_fix_to_float<<<nblk(n, 256), 256, 0, c->stream>>>(c->rho_fx, c->rho, n);
  c->launches++;
  return tild_check(c, cudaGetLastError(), "spread") ? TILD_ERR_CUDA : TILD_OK;
}

int tild_run_forces(tild_ctx* c, int64_t step, bool integrate, float* f_bead) {
  if (integrate && c->sort_interval > 0 && step - 1 - c->last_sort_step >= c->sort_interval) {
    tild_mark(c, STAGE_SORT);
    int rs = tild_sort_beads(c);
    if (rs) return rs;
  }
  int rc = tild_run_spread(c);
  if (rc) return rc;
  tild_mark(c, STAGE_R2C);
  if (tild_check_fft(c, cufftExecR2C(c->plan_r2c, c->rho, c->rhok), "R2C")) return TILD_ERR_CUDA;
  if (c->T > 0 && (c->styles_k.size() > 0 || c->C)) {
    KArgs ka;
    ka.nstyle = (int)c->styles_k.size();
    for (int s = 0; s < ka.nstyle; s++) {
      ka.a[s] = c->styles_k[s].a;
      ka.b[s] = c->styles_k[s].b;
      ka.scale[s] = (float)tild_ramp_ratio(c, s, step);
    }
    tild_mark(c, STAGE_KMUL);
    if (c->D == 3) launch_kmul<3>(c, ka);
    else launch_kmul<2>(c, ka);
    c->launches++;
    if (tild_check(c, cudaGetLastError(), "kmul")) return TILD_ERR_CUDA;
    tild_mark(c, STAGE_C2R);
    if (tild_check_fft(c, cufftExecC2R(c->plan_c2r, c->gk, c->gfield), "C2R")) return TILD_ERR_CUDA;
  } else {
    if (tild_check(c, cudaMemsetAsync(c->gfield, 0, sizeof(float) * (size_t)(c->T + c->C) * c->D * c->g.M, c->stream),
                   "zero field"))
      return TILD_ERR_CUDA;
  }
  if (!c->fields.empty()) tild_mark(c, STAGE_FIELD);
  for (size_t fi = 0; fi < c->fields.size(); fi++) {
    k_fieldphase_apply<<<nblk(c->g.M, 256), 256, 0, c->stream>>>(c->gfield, c->rho,
                                                                 c->frfield + (long long)fi * c->D * c->g.M,
                                                                 c->fields[fi].a, c->fields[fi].b, c->D, c->g.M);
    c->launches++;
  }
  GArgs ga;
  memset(&ga, 0, sizeof(ga));
  ga.step = step;
  ga.seed = c->cfg.seed;
  ga.delt = c->cfg.delt;
  ga.noise_mag = c->cfg.noise_mag;
  ga.n_integ = c->cfg.n_integrators;
  for (int k = 0; k < ga.n_integ; k++) ga.integ_kind[k] = c->cfg.integrators[k].kind;
  for (int t = 0; t < c->T; t++) {
    ga.type_mask[t] = c->type_integ_mask[t];
    ga.mass[t] = c->cfg.mass[t];
    ga.diff[t] = c->cfg.diff[t];
  }
  for (int b = 0; b < c->cfg.n_bond_types; b++) {
    ga.bond_k[b] = c->cfg.bond_k[b];
    ga.bond_req[b] = c->cfg.bond_req[b];
  }
  tild_mark(c, STAGE_GATHER);
  k_interleave<<<nblk(c->g.M, 256), 256, 0, c->stream>>>(c->gfield, c->g4, c->T + c->C, c->D, c->g.M);
  c->launches++;
  if (c->D == 3) dispatch_p_gather<3>(c, ga, integrate, f_bead);
  else dispatch_p_gather<2>(c, ga, integrate, f_bead);
  c->launches++;
  if (tild_check(c, cudaGetLastError(), "gather")) return TILD_ERR_CUDA;
  if (integrate) c->cur ^= 1;
  c->forces_step = step;
  c->have_forces = true;
  return TILD_OK;
}
