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

namespace {

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// ---------------------------------------------------------------------------------------------
// Spreading: d_charge_grid / d_charge_grid_charges (device_grid_utils.cu:111-343)
// ---------------------------------------------------------------------------------------------
template <int D, int P>
__global__ void __launch_bounds__(256) k_spread(const float4* __restrict__ pos, const float* __restrict__ charge, int ns,
                                               Geom g, float* __restrict__ rho, int T, int C, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const float4 p = pos[i];
  const float xs[3] = {p.x, p.y, p.z};
  if (!isfinite(p.x) || !isfinite(p.y) || (D == 3 && !isfinite(p.z))) {
    atomicOr(status, ST_NONFINITE_POS);
    return;
  }
  const int t = tild_type_of(p.w);
  float W[3][P + 1];
  int idx[3][P + 1];
#pragma unroll
  for (int d = 0; d < D; d++) {
    const int b = axis_base<P>(xs[d], g.dx[d], W[d]);
#pragma unroll
    for (int a = 0; a <= P; a++) idx[d][a] = wrap_idx(b + a, g.nx[d], status);
  }
  float* rt = rho + (long long)t * g.M;
  const float q = C ? charge[i] : 0.f;
  float* rc = rho + (long long)T * g.M;
  if (D == 3) {
#pragma unroll
    for (int ix = 0; ix <= P; ix++)
#pragma unroll
      for (int iy = 0; iy <= P; iy++) {
        const long long row = idx[0][ix] + (long long)idx[1][iy] * g.nx[0];
#pragma unroll
        for (int iz = 0; iz <= P; iz++) {
          const long long m = row + (long long)idx[2][iz] * g.nx[1] * g.nx[0];
          const float W3 = W[0][ix] * W[1][iy] * W[2][iz] / g.gvol;
          atomicAdd(rt + m, W3);
          if (C && q != 0.f) atomicAdd(rc + m, W3 * q);
        }
      }
  } else {
#pragma unroll
    for (int ix = 0; ix <= P; ix++)
#pragma unroll
      for (int iy = 0; iy <= P; iy++) {
        const long long m = (long long)idx[1][iy] * g.nx[0] + idx[0][ix];
        const float W3 = W[0][ix] * W[1][iy] / g.gvol;
        atomicAdd(rt + m, W3);
        if (C && q != 0.f) atomicAdd(rc + m, W3 * q);
      }
  }
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

template <int D, int P, bool INTEG, bool XW>
__global__ void __launch_bounds__(256) k_gather(const float4* __restrict__ pos_in, float4* __restrict__ pos_io,
                                               float* __restrict__ noise, const int* __restrict__ bead_id,
                                               const int* __restrict__ bond_nbr, const int* __restrict__ bond_info,
                                               const float* __restrict__ charge, const float* __restrict__ gfield,
                                               Geom g, int T, int C, GArgs ga, float* __restrict__ f_out,
                                               curandStateXORWOW_t* __restrict__ xw, int ns, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const float4 p = pos_in[i];
  float x[3] = {p.x, p.y, p.z};
  const bool finite = isfinite(p.x) && isfinite(p.y) && (D == 2 || isfinite(p.z));
  float f[3] = {0.f, 0.f, 0.f};
  const int t = tild_type_of(p.w);
  if (finite) {
    float W[3][P + 1];
    int idx[3][P + 1];
#pragma unroll
    for (int d = 0; d < D; d++) {
      const int b = axis_base<P>(x[d], g.dx[d], W[d]);
#pragma unroll
      for (int a = 0; a <= P; a++) idx[d][a] = wrap_idx(b + a, g.nx[d], status);
    }
    const long long M = g.M;
    const float* G0 = gfield + (long long)t * D * M;
    if (C) {
      const float q = charge[i];
      if (q != 0.f) {
        const float* E0 = gfield + (long long)T * D * M;
        float e[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int ix = 0; ix <= P; ix++)
#pragma unroll
          for (int iy = 0; iy <= P; iy++) {
            const long long row = idx[0][ix] + (long long)idx[1][iy] * g.nx[0];
            if (D == 3) {
#pragma unroll
              for (int iz = 0; iz <= P; iz++) {
                const long long m = row + (long long)idx[2][iz] * g.nx[1] * g.nx[0];
                const float w = W[0][ix] * W[1][iy] * W[2][iz];
#pragma unroll
                for (int d = 0; d < D; d++) e[d] += E0[d * M + m] * w;
              }
            } else {
              const float w = W[0][ix] * W[1][iy];
#pragma unroll
              for (int d = 0; d < D; d++) e[d] += E0[d * M + row] * w;
            }
          }
#pragma unroll
        for (int d = 0; d < D; d++) f[d] += e[d] * q;
      }
    }
#pragma unroll
    for (int ix = 0; ix <= P; ix++)
#pragma unroll
      for (int iy = 0; iy <= P; iy++) {
        const long long row = idx[0][ix] + (long long)idx[1][iy] * g.nx[0];
        if (D == 3) {
#pragma unroll
          for (int iz = 0; iz <= P; iz++) {
            const long long m = row + (long long)idx[2][iz] * g.nx[1] * g.nx[0];
            const float w = W[0][ix] * W[1][iy] * W[2][iz];
#pragma unroll
            for (int d = 0; d < D; d++) f[d] += G0[d * M + m] * w;
          }
        } else {
          const float w = W[0][ix] * W[1][iy];
#pragma unroll
          for (int d = 0; d < D; d++) f[d] += G0[d * M + row] * w;
        }
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
  } else {
    atomicOr(status, ST_NONFINITE_POS);
  }
  const int bid = bead_id[i];
  if (f_out) {
#pragma unroll
    for (int d = 0; d < D; d++) f_out[(long long)bid * D + d] = f[d];
  }
  if (!INTEG) return;
  // integrators in input order (integrator.cu:24-39 is called for each in turn)
  const int mask = ga.type_mask[t];
  float4 po = pos_io[i];  // x_{n-1} (GJF xo)
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
  k_spread<D, P><<<nblk(c->ns, 256), 256, 0, c->stream>>>(c->pos[c->cur], c->charge, c->ns, c->g, c->rho, c->T, c->C,
                                                           c->d_status);
}

template <int D, int P>
void launch_gather(tild_ctx* c, const GArgs& ga, bool integ, float* f_out) {
  const float4* pin = c->pos[c->cur];
  float4* pio = c->pos[c->cur ^ 1];
  const unsigned nb = nblk(c->ns, 256);
  const bool xw = c->cfg.rng == TILD_RNG_XORWOW;
  if (integ) {
    if (xw)
      k_gather<D, P, true, true><<<nb, 256, 0, c->stream>>>(pin, pio, c->noise, c->bead_id, c->bond_nbr, c->bond_info,
                                                            c->charge, c->gfield, c->g, c->T, c->C, ga, f_out, c->xorwow,
                                                            c->ns, c->d_status);
    else
      k_gather<D, P, true, false><<<nb, 256, 0, c->stream>>>(pin, pio, c->noise, c->bead_id, c->bond_nbr, c->bond_info,
                                                             c->charge, c->gfield, c->g, c->T, c->C, ga, f_out,
                                                             c->xorwow, c->ns, c->d_status);
  } else {
    k_gather<D, P, false, false><<<nb, 256, 0, c->stream>>>(pin, pio, c->noise, c->bead_id, c->bond_nbr, c->bond_info,
                                                            c->charge, c->gfield, c->g, c->T, c->C, ga, f_out,
                                                            c->xorwow, c->ns, c->d_status);
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
  tild_mark(c, STAGE_ZERO);
  if (tild_check(c, cudaMemsetAsync(c->rho, 0, sizeof(float) * (size_t)(c->T + c->C) * c->g.M, c->stream), "zero rho"))
    return TILD_ERR_CUDA;
  tild_mark(c, STAGE_SPREAD);
  if (c->D == 3) dispatch_p_spread<3>(c);
  else dispatch_p_spread<2>(c);
  c->launches++;
  return tild_check(c, cudaGetLastError(), "spread") ? TILD_ERR_CUDA : TILD_OK;
}

int tild_run_forces(tild_ctx* c, int64_t step, bool integrate, float* f_bead) {
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
  if (c->D == 3) dispatch_p_gather<3>(c, ga, integrate, f_bead);
  else dispatch_p_gather<2>(c, ga, integrate, f_bead);
  c->launches++;
  if (tild_check(c, cudaGetLastError(), "gather")) return TILD_ERR_CUDA;
  if (integrate) c->cur ^= 1;
  c->forces_step = step;
  c->have_forces = true;
  return TILD_OK;
}
