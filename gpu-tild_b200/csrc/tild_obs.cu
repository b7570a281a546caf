// tild_obs.cu — observables (FP64 device reductions), avg_sk accumulation, stencil export and
// the cell / neighbour list.
//
// calc_properties() in the reference (calc_properties.cu:20-116) evaluates every energy and
// virial term in real space with one more IFFT each, copies M floats to the host and sums
// them in FP32 (integ_utils.cu:3-13).  Here each term is a k-space inner product over the R2C
// half spectrum (Parseval), reduced in FP64 on the device:
//   E_s  = dV * sum_full u_s(k) rho_b(k) conj(rho_a(k)) / M           (pair_style.cu:204-233)
//   P_s  = dV/(V D) * sum_full vir_s(k) rho_b(k) conj(rho_a(k)) / M     (pair_style.cu:235-260)
//   E_el = sum_full 4 pi lB e^{-k^2/(2a^2)} / k^2 |rho_c(k)|^2 / M      (calc_properties.cu:106-116)
// with sum_full = sum_half w(k) Re(...), w = 1 on the kx = 0 and Nyquist planes, else 2.
#include "tild_internal.cuh"
#include <cmath>

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kObsThreads = 256;

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

__device__ __forceinline__ double hermitian_weight(int ix, int nx0) {
  return (ix == 0 || ((nx0 % 2 == 0) && ix == nx0 / 2)) ? 1.0 : 2.0;
}

// Block-wide sum of NV doubles per thread; thread 0 writes the block's partials.
template <int NV>
__device__ void block_sum_write(double (&v)[NV], double* out) {
  __shared__ double sh[NV][kObsThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double s = 0.0;
      for (int w = 0; w < kObsThreads / 32; w++) s += sh[k][w];
      out[(long long)blockIdx.x * NV + k] = s;
    }
  }
}

// one FFT pair style: energy and nP virial components
__global__ void __launch_bounds__(kObsThreads) k_obs_style(const float2* __restrict__ rhok, const float* __restrict__ ut,
                                                          const float2* __restrict__ vk, int a, int b, Geom g, int nP,
                                                          double scale, double* __restrict__ partial) {
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  const long long Mh = g.Mh;
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < Mh; h += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(h % g.nxh);
    const double w = hermitian_weight(ix, g.nx[0]);
    const float2 ra = rhok[(long long)a * Mh + h], rb = rhok[(long long)b * Mh + h];
    // rho_b conj(rho_a)
    const double re = (double)rb.x * ra.x + (double)rb.y * ra.y;
    const double im = (double)rb.y * ra.x - (double)rb.x * ra.y;
    v[0] += w * (double)ut[h] * scale * re;
    for (int j = 0; j < nP; j++) {
      const float2 q = vk[(long long)j * Mh + h];
      v[1 + j] += w * ((double)q.x * re - (double)q.y * im);
    }
  }
  block_sum_write<7>(v, partial);
}

// smeared electrostatics: psi_k = 4 pi lB e^{-k^2/(2 a^2)} rho_c(k) / (M k^2), E = sum_r psi rho_c
__global__ void __launch_bounds__(kObsThreads) k_obs_charge(const float2* __restrict__ rc, const float* __restrict__ kk,
                                                           Geom g, int D, double lB, double a2,
                                                           double* __restrict__ partial) {
  double v[1] = {0.0};
  const long long Mh = g.Mh;
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < Mh; h += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(h % g.nxh);
    const long long r = h / g.nxh;
    const int iy = (int)(r % g.nx[1]);
    const int iz = (int)(r / g.nx[1]);
    const int nn[3] = {ix, iy, iz};
    double k2 = 0.0;
    int off = 0;
    for (int d = 0; d < D; d++) {
      const int N = g.nx[d];
      const int sf = ((float)nn[d] < (float)N / 2.0f) ? nn[d] : nn[d] - N;
      const double kd = 2.0 * kPi * (double)sf / (double)g.L[d];
      k2 += kd * kd;
      off += N;
    }
    (void)kk;
    if (k2 == 0.0) continue;
    const float2 c = rc[h];
    const double m2 = (double)c.x * c.x + (double)c.y * c.y;
    v[0] += hermitian_weight(ix, g.nx[0]) * 4.0 * kPi * lB / k2 * exp(-k2 / (2.0 * a2)) * m2;
  }
  block_sum_write<1>(v, partial);
}

// host_bonds (bonds.cu:3-52): every bond once (partner id >= own id), FP64 accumulation
__global__ void __launch_bounds__(kObsThreads) k_obs_bonds(const float4* __restrict__ pos, const int* __restrict__ bead_id,
                                                          const int* __restrict__ nbr, const int* __restrict__ info,
                                                          const float* __restrict__ bk, const float* __restrict__ br,
                                                          Geom g, int D, int slot0, int nslot,
                                                          double* __restrict__ partial) {
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = slot0 + blockIdx.x * blockDim.x + threadIdx.x; i < slot0 + nslot; i += gridDim.x * blockDim.x) {
    const int id1 = bead_id[i];
    if (id1 < 0) continue;
    const int in = info[i], nb = in & 3;
    const float4 p = pos[i];
    const float x1[3] = {p.x, p.y, p.z};
    for (int b = 0; b < nb; b++) {
      const int j = nbr[3 * i + b];
      if (bead_id[j] < id1) continue;
      const int bt = (in >> (8 + 8 * b)) & 0xff;
      const float4 q = pos[j];
      const float x2[3] = {q.x, q.y, q.z};
      double dr[3] = {0, 0, 0}, mdr2 = 0.0;
      for (int d = 0; d < D; d++) {
        const float drf = x1[d] - x2[d];
        double dv = (double)x1[d] - (double)x2[d];
        if (drf > g.Lh[d]) dv -= (double)g.L[d];
        else if (drf < -g.Lh[d]) dv += (double)g.L[d];
        dr[d] = dv;
        mdr2 += dv * dv;
      }
      const double mdr = sqrt(mdr2), delr = mdr - (double)br[bt];
      v[0] += delr * delr * (double)bk[bt];
      const double mf = 2.0 * (double)bk[bt] * delr / mdr;
      v[1] += -mf * dr[0] * dr[0];
      v[2] += -mf * dr[1] * dr[1];
      if (D == 2) {
        v[3] += -mf * dr[0] * dr[1];
      } else {
        v[3] += -mf * dr[2] * dr[2];
        v[4] += -mf * dr[0] * dr[1];
        v[5] += -mf * dr[0] * dr[2];
        v[6] += -mf * dr[1] * dr[2];
      }
    }
  }
  block_sum_write<7>(v, partial);
}

// avg_sk: acc += rho_k * rho_k / M (Compute.cu:89-109 multiplies rho_k by itself, no conjugate)
__global__ void k_sk_acc(double2* __restrict__ acc, const float2* __restrict__ rk, long long Mh, double invM) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= Mh) return;
  const float2 c = rk[h];
  const double re = (double)c.x * c.x - (double)c.y * c.y, im = 2.0 * (double)c.x * c.y;
  double2 a = acc[h];
  a.x += re * invM;
  a.y += im * invM;
  acc[h] = a;
}

// stencil export in d_charge_grid order (device_grid_utils.cu:305-339)
template <int D, int P>
__global__ void k_stencil(const float4* __restrict__ pos, const int* __restrict__ bead_id, Geom g, int slot0, int nslot,
                          int* __restrict__ inds, float* __restrict__ wout, int* status) {
  const int i = slot0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= slot0 + nslot || bead_id[i] < 0) return;
  const float4 p = pos[i];
  const float xs[3] = {p.x, p.y, p.z};
  float W[3][P + 1];
  int idx[3][P + 1];
  for (int d = 0; d < D; d++) {
    const int b = axis_base<P>(xs[d], g.dx[d], W[d]);
    for (int a = 0; a <= P; a++) idx[d][a] = wrap_idx(b + a, g.nx[d], status);
  }
  constexpr int S = (D == 3) ? (P + 1) * (P + 1) * (P + 1) : (P + 1) * (P + 1);
  const long long o = (long long)bead_id[i] * S;
  int ct = 0;
  for (int ix = 0; ix <= P; ix++)
    for (int iy = 0; iy <= P; iy++) {
      if (D == 3) {
        for (int iz = 0; iz <= P; iz++) {
          if (inds) inds[o + ct] = idx[0][ix] + (idx[1][iy] + idx[2][iz] * g.nx[1]) * g.nx[0];
          if (wout) wout[o + ct] = W[0][ix] * W[1][iy] * W[2][iz] / g.gvol;
          ct++;
        }
      } else {
        if (inds) inds[o + ct] = idx[1][iy] * g.nx[0] + idx[0][ix];
        if (wout) wout[o + ct] = W[0][ix] * W[1][iy] / g.gvol;
        ct++;
      }
    }
}

// ---- neighbour list (nlist.cu:64-228) -----------------------------------------------------------
struct CellGeom {
  int nc[3];
  float Lc[3];
  int total, cmax, D;
};

__device__ __forceinline__ int cell_index(const CellGeom& cg, int c0, int c1, int c2) {
  return (cg.D == 2) ? c0 + cg.nc[0] * c1 : c0 + (c1 + c2 * cg.nc[1]) * cg.nc[0];
}

// d_assign_cells: cell = int(x / Lcell) per axis (cells are folded back into range for x == L)
__global__ void k_assign_cells(const float4* __restrict__ pos, const int* __restrict__ bead_id, CellGeom cg, int ns,
                               int group_type, int* __restrict__ cell_of_slot, int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const float4 p = pos[i];
  if (bead_id[i] < 0 || (group_type >= 0 && tild_type_of(p.w) != group_type)) {
    cell_of_slot[i] = -1;
    return;
  }
  const float xs[3] = {p.x, p.y, p.z};
  int c[3] = {0, 0, 0};
  for (int j = 0; j < cg.D; j++) {
    int v = (int)(xs[j] / cg.Lc[j]);
    if (v >= cg.nc[j]) v -= cg.nc[j];
    if (v < 0) v += cg.nc[j];
    c[j] = v;
  }
  const int cn = cell_index(cg, c[0], c[1], c[2]);
  cell_of_slot[i] = cn;
  atomicAdd(cnt + cn, 1);
}

__global__ void k_fill_cells(const int* __restrict__ cell_of_slot, int ns, int* __restrict__ cursor,
                             int* __restrict__ cell_slots, int cmax, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const int cn = cell_of_slot[i];
  if (cn < 0) return;
  const int k = atomicAdd(cursor + cn, 1);
  if (k < cmax) cell_slots[(long long)cn * cmax + k] = i;
  else atomicOr(status, ST_NLIST_OVERFLOW);
}

// d_make_nlist: 27 (9 in 2D) cells with the reference's +-1 wrap; the bead itself is listed
// (mdr2 = 0 < rc^2, as in the reference).  Each row is sorted by bead id afterwards.
__global__ void k_make_nlist(const float4* __restrict__ pos, const int* __restrict__ bead_id, CellGeom cg, int ns,
                             const int* __restrict__ cell_of_slot, const int* __restrict__ cnt,
                             const int* __restrict__ cell_slots, float rc2, Geom g, int* __restrict__ ncount,
                             int* __restrict__ neigh, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const int cn = cell_of_slot[i];
  const int bid = bead_id[i];
  if (bid < 0) return;
  if (cn < 0) {
    ncount[bid] = 0;
    return;
  }
  int nn[3];
  if (cg.D == 2) { nn[1] = cn / cg.nc[0]; nn[0] = cn % cg.nc[0]; nn[2] = 1; }
  else {
    nn[2] = cn / (cg.nc[1] * cg.nc[0]);
    const int r = cn - nn[2] * cg.nc[0] * cg.nc[1];
    nn[1] = r / cg.nc[0];
    nn[0] = r % cg.nc[0];
  }
  const float4 p = pos[i];
  const float xi[3] = {p.x, p.y, p.z};
  int* row = neigh + (long long)bid * cg.cmax;
  int ct = 0;
  for (int ix = nn[0] - 1; ix <= nn[0] + 1; ix++) {
    int nix = ix;
    if (nix < 0) nix = cg.nc[0] - 1;
    else if (nix == cg.nc[0]) nix = 0;
    for (int iy = nn[1] - 1; iy <= nn[1] + 1; iy++) {
      int niy = iy;
      if (niy < 0) niy = cg.nc[1] - 1;
      else if (niy == cg.nc[1]) niy = 0;
      for (int iz = nn[2] - 1; iz <= nn[2] + 1; iz++) {
        int niz = iz;
        if (cg.D == 2) niz = 0;
        else {
          if (niz < 0) niz = cg.nc[2] - 1;
          else if (niz == cg.nc[2]) niz = 0;
        }
        const int ncn = cell_index(cg, nix, niy, niz);
        const int cc = min(cnt[ncn], cg.cmax);
        for (int q = 0; q < cc; q++) {
          const int js = cell_slots[(long long)ncn * cg.cmax + q];
          const float4 pj = pos[js];
          const float xj[3] = {pj.x, pj.y, pj.z};
          float mdr2 = 0.f;
          for (int j = 0; j < cg.D; j++) {
            float dr = xi[j] - xj[j];
            if (dr < -g.Lh[j]) dr += g.L[j];
            else if (dr > g.Lh[j]) dr -= g.L[j];
            mdr2 += dr * dr;
          }
          if (mdr2 < rc2) {
            if (ct < cg.cmax) row[ct] = bead_id[js];
            else atomicOr(status, ST_NLIST_OVERFLOW);
            ct++;
          }
        }
        if (cg.D == 2) break;
      }
    }
  }
  const int n = min(ct, cg.cmax);
  for (int a = 1; a < n; a++) {  // insertion sort of the row
    const int v = row[a];
    int b = a - 1;
    while (b >= 0 && row[b] > v) {
      row[b + 1] = row[b];
      b--;
    }
    row[b + 1] = v;
  }
  ncount[bid] = ct;
}

__global__ void k_scatter_int(const int* __restrict__ src_slot, const int* __restrict__ bead_id, int ns,
                              int* __restrict__ dst_bead) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns || bead_id[i] < 0) return;
  dst_bead[bead_id[i]] = src_slot[i];
}

}  // namespace

int tild_ensure_red(tild_ctx* c, int nvals, int nblocks) {
  const int need = nvals * nblocks;
  if (need <= c->red_cap) return TILD_OK;
  cudaFree(c->red);
  c->red = nullptr;
  c->red_cap = 0;
  if (tild_check(c, cudaMalloc(&c->red, sizeof(double) * need), "alloc reduction scratch")) return TILD_ERR_OOM;
  c->red_cap = need;
  return TILD_OK;
}

static int reduce_host(tild_ctx* c, int nvals, int nblocks, double* out) {
  std::vector<double> h((size_t)nvals * nblocks);
  if (tild_check(c, cudaMemcpyAsync(h.data(), c->red, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream),
                 "copy partials") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync partials"))
    return TILD_ERR_CUDA;
  for (int k = 0; k < nvals; k++) out[k] = 0.0;
  for (int b = 0; b < nblocks; b++)
    for (int k = 0; k < nvals; k++) out[k] += h[(size_t)b * nvals + k];
  return TILD_OK;
}

int tild_obs_compute(tild_ctx* c, int si, tild_obs* o) {
  const SysHost& h = c->sys[si];
  const SysDev& hd = c->h_sys[si];
  memset(o, 0, sizeof(*o));
  o->n_styles = h.cfg.n_styles;
  o->n_p_comps = h.nP;
  o->step = h.forces_step;
  const int nblocks = 296;
  if (tild_ensure_red(c, 7, nblocks)) return TILD_ERR_OOM;
  const float2* rk = tild_half_spectra(c, si);  // per-channel half spectra of the last force evaluation
  double upe = 0.0;
  for (size_t k = 0; k < h.fft_cfg.size(); k++) {
    const int ci = h.fft_cfg[k];
    const double scale = ramp_ratio(hd, (int)k, h.forces_step);
    k_obs_style<<<nblocks, kObsThreads, 0, c->stream>>>(rk, c->utab + h.utab0 + (long long)k * h.g.Mh,
                                                         reinterpret_cast<const float2*>(c->virk) + h.virk0 +
                                                             (long long)k * h.nP * h.g.Mh,
                                                         hd.sa[k], hd.sb[k], h.g, h.nP, scale, c->red);
    c->launches++;
    double r[7];
    if (reduce_host(c, 7, nblocks, r)) return TILD_ERR_CUDA;
    o->style_energy[ci] = r[0] * h.dV;
    upe += o->style_energy[ci];
    for (int j = 0; j < h.nP; j++) {
      o->style_virial[ci][j] = r[1 + j] * h.dV / h.V / (double)h.D;
      o->ptens[j] += o->style_virial[ci][j];
    }
  }
  if (h.C) {
    k_obs_charge<<<nblocks, kObsThreads, 0, c->stream>>>(rk + (long long)h.T * h.g.Mh, c->kk + h.kd0, h.g, h.D,
                                                          (double)h.cfg.bjerrum,
                                                          (double)h.cfg.smearing * (double)h.cfg.smearing, c->red);
    c->launches++;
    double r[1];
    if (reduce_host(c, 1, nblocks, r)) return TILD_ERR_CUDA;
    o->uelec = r[0] / (double)h.g.M;
    upe += o->uelec;
  }
  {
    const SysDev* dsys = c->d_sys + si;
    k_obs_bonds<<<nblocks, kObsThreads, 0, c->stream>>>(c->pos[c->cur], c->bead_id, c->bond_nbr, c->bond_info,
                                                         dsys->bond_k, dsys->bond_req, h.g, h.D, h.slot0, h.ns_pad,
                                                         c->red);
    c->launches++;
    double r[7];
    if (reduce_host(c, 7, nblocks, r)) return TILD_ERR_CUDA;
    o->ubond = r[0];
    upe += o->ubond;
    for (int j = 0; j < h.nP; j++) {
      o->bond_vir[j] = r[1 + j] * (1.0 / h.V / (double)h.D);
      o->ptens[j] += o->bond_vir[j];
    }
  }
  o->upe = upe;
  return tild_check(c, cudaGetLastError(), "observables") ? TILD_ERR_CUDA : TILD_OK;
}

int tild_sk_acc_run(tild_ctx* c, int si, int slot, int type) {
  SysHost& h = c->sys[si];
  if (!h.sk[slot]) {
    if (tild_check(c, cudaMalloc(&h.sk[slot], sizeof(double2) * h.g.Mh), "alloc sk")) return TILD_ERR_OOM;
    if (tild_check(c, cudaMemsetAsync(h.sk[slot], 0, sizeof(double2) * h.g.Mh, c->stream), "zero sk"))
      return TILD_ERR_CUDA;
    h.sk_calls[slot] = 0;
  }
  k_sk_acc<<<nblk(h.g.Mh, 256), 256, 0, c->stream>>>(reinterpret_cast<double2*>(h.sk[slot]),
                                                      tild_half_spectra(c, si) + (long long)type * h.g.Mh, h.g.Mh,
                                                      1.0 / (double)h.g.M);
  c->launches++;
  h.sk_calls[slot]++;
  return tild_check(c, cudaGetLastError(), "sk accumulate") ? TILD_ERR_CUDA : TILD_OK;
}

template <int D, int P>
static void launch_stencil(tild_ctx* c, const SysHost& h, int* inds, float* w) {
  k_stencil<D, P><<<nblk(h.ns_pad, 256), 256, 0, c->stream>>>(c->pos[c->cur], c->bead_id, h.g, h.slot0, h.ns_pad,
                                                               inds, w, c->d_status);
}

int tild_stencil_run(tild_ctx* c, int si, int* inds_dev, float* w_dev) {
  const SysHost& h = c->sys[si];
  if (c->D == 3) {
    switch (c->P) {
      case 0: launch_stencil<3, 0>(c, h, inds_dev, w_dev); break;
      case 1: launch_stencil<3, 1>(c, h, inds_dev, w_dev); break;
      case 2: launch_stencil<3, 2>(c, h, inds_dev, w_dev); break;
      case 3: launch_stencil<3, 3>(c, h, inds_dev, w_dev); break;
      default: launch_stencil<3, 4>(c, h, inds_dev, w_dev); break;
    }
  } else {
    switch (c->P) {
      case 0: launch_stencil<2, 0>(c, h, inds_dev, w_dev); break;
      case 1: launch_stencil<2, 1>(c, h, inds_dev, w_dev); break;
      case 2: launch_stencil<2, 2>(c, h, inds_dev, w_dev); break;
      case 3: launch_stencil<2, 3>(c, h, inds_dev, w_dev); break;
      default: launch_stencil<2, 4>(c, h, inds_dev, w_dev); break;
    }
  }
  c->launches++;
  return tild_check(c, cudaGetLastError(), "stencil") ? TILD_ERR_CUDA : TILD_OK;
}

// NList::Initialize geometry (nlist.cu:85-102) in FP32 as the reference computes it
int tild_nlist_geom(const SysHost& h, float rc, int* nc, float* Lc, int* total, int* cmax) {
  float cell_vol = 1.0f, V = 1.0f;
  *total = 1;
  for (int j = 0; j < 3; j++) { nc[j] = 1; Lc[j] = 1.f; }
  for (int j = 0; j < h.D; j++) {
    nc[j] = (int)(h.g.L[j] / rc);
    if (nc[j] < 1) return TILD_ERR_BAD_INPUT;
    Lc[j] = h.g.L[j] / (int)nc[j];
    *total *= nc[j];
    cell_vol *= Lc[j];
    V *= h.g.L[j];
  }
  *cmax = (int)((float)(h.ns * cell_vol / V) * 7.5);
  return TILD_OK;
}

int tild_nlist_run(tild_ctx* c, int si, float rc, int group_type, int* cell_of_bead_dev, int* ncount_dev,
                   int* neigh_dev) {
  const SysHost& h = c->sys[si];
  CellGeom cg;
  cg.D = h.D;
  if (tild_nlist_geom(h, rc, cg.nc, cg.Lc, &cg.total, &cg.cmax)) return TILD_ERR_BAD_INPUT;
  if (cg.cmax < 1) return TILD_ERR_BAD_INPUT;
  int *cell_of_slot = nullptr, *cnt = nullptr, *cursor = nullptr, *cell_slots = nullptr;
  int rc_ = TILD_OK;
  const int n = h.ns_pad;
  const float4* pos = c->pos[c->cur] + h.slot0;
  const int* bid = c->bead_id + h.slot0;
  if (tild_check(c, cudaMalloc(&cell_of_slot, sizeof(int) * n), "alloc nlist") ||
      tild_check(c, cudaMalloc(&cnt, sizeof(int) * cg.total), "alloc nlist") ||
      tild_check(c, cudaMalloc(&cursor, sizeof(int) * cg.total), "alloc nlist") ||
      tild_check(c, cudaMalloc(&cell_slots, sizeof(int) * (size_t)cg.total * cg.cmax), "alloc nlist"))
    rc_ = TILD_ERR_OOM;
  if (rc_ == TILD_OK) {
    cudaMemsetAsync(cnt, 0, sizeof(int) * cg.total, c->stream);
    cudaMemsetAsync(cursor, 0, sizeof(int) * cg.total, c->stream);
    k_assign_cells<<<nblk(n, 256), 256, 0, c->stream>>>(pos, bid, cg, n, group_type, cell_of_slot, cnt);
    k_fill_cells<<<nblk(n, 256), 256, 0, c->stream>>>(cell_of_slot, n, cursor, cell_slots, cg.cmax, c->d_status);
    k_make_nlist<<<nblk(n, 256), 256, 0, c->stream>>>(pos, bid, cg, n, cell_of_slot, cnt, cell_slots, rc * rc, h.g,
                                                      ncount_dev, neigh_dev, c->d_status);
    c->launches += 3;
    k_scatter_int<<<nblk(n, 256), 256, 0, c->stream>>>(cell_of_slot, bid, n, cell_of_bead_dev);
    c->launches++;
    if (tild_check(c, cudaStreamSynchronize(c->stream), "nlist")) rc_ = TILD_ERR_CUDA;
  }
  cudaFree(cell_of_slot);
  cudaFree(cnt);
  cudaFree(cursor);
  cudaFree(cell_slots);
  return rc_;
}
