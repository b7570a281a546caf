// tild_api.cu — the C ABI declared in include/tild.h.
//
// Setup mirrors initialize() (initialize.cu:20-244): geometry in FP32 as the reference computes
// it, device allocation, k-space tables, the cuFFT plans.  The per-step entry points wrap the
// kernels of tild_step.cu and tild_obs.cu.  Errors never exit the process: every call returns
// a tild_status and records a message on the context.
#include "tild_internal.cuh"
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>

namespace {

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

int set_err(tild_ctx* c, int code, const char* msg) {
  if (c) c->err = msg;
  return code;
}

// pack positions [ns][D] (bead order) of one system into float4 slots with the type in .w
__global__ void k_pack_pos(const float* __restrict__ x, const int* __restrict__ types, const int* __restrict__ slot_of,
                           int ns, int D, float4* __restrict__ pos) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= ns) return;
  const float* xb = x + (long long)b * D;
  pos[slot_of[b]] = make_float4(xb[0], xb[1], D == 3 ? xb[2] : 0.f, __int_as_float(types[b] & 0xff));
}

__global__ void k_fill_padding(float4* __restrict__ p0, float4* __restrict__ p1, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float4 pad = make_float4(0.f, 0.f, 0.f, __int_as_float(kPadType));
  p0[s] = pad;
  p1[s] = pad;
}

// flag[0] |= 1 when any of the n uploaded values is not finite
__global__ void k_check_finite(const float* __restrict__ v, long long n, int* __restrict__ flag) {
  bool bad = false;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(v[k]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

__global__ void k_pack_noise(const float* __restrict__ src, const int* __restrict__ slot_of, int ns, int D,
                             float* __restrict__ noise) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= ns) return;
  const int s = slot_of[b];
  for (int d = 0; d < 3; d++) noise[3 * (long long)s + d] = (src && d < D) ? src[(long long)b * D + d] : 0.f;
}

__global__ void k_unpack_pos(const float4* __restrict__ pos, const int* __restrict__ bead_id, int n, int D,
                             float* __restrict__ x) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n || bead_id[s] < 0) return;
  const float4 p = pos[s];
  float* xb = x + (long long)bead_id[s] * D;
  xb[0] = p.x;
  xb[1] = p.y;
  if (D == 3) xb[2] = p.z;
}

__global__ void k_unpack_noise(const float* __restrict__ noise, const int* __restrict__ bead_id, int n, int D,
                               float* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n || bead_id[s] < 0) return;
  for (int d = 0; d < D; d++) out[(long long)bead_id[s] * D + d] = noise[3 * (long long)s + d];
}

__global__ void k_init_xorwow(curandStateXORWOW_t* st, const int* __restrict__ bead_id, int n, unsigned int seed) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n || bead_id[s] < 0) return;
  // init_dev_rng (cuda_random_posits.cu:22-30): curand_init(seed, bead, 0)
  curand_init(seed, (unsigned long long)bead_id[s], 0, &st[s]);
}

template <typename T>
int dalloc(tild_ctx* c, T** p, size_t n, const char* what) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    c->err = std::string("device allocation failed: ") + what + " (" + cudaGetErrorString(e) + ")";
    return TILD_ERR_OOM;
  }
  return TILD_OK;
}

void free_all(tild_ctx* c) {
  void* ptrs[] = {c->pos[0], c->pos[1], c->noise, c->bead_id, c->slot_of, c->bond_nbr, c->bond_info, c->charge,
                  c->types_dev, c->xorwow, c->rho, c->rhok, c->gk, c->gfield, c->utab, c->ctab, c->virk, c->frfield,
                  c->rho_fx, c->g4, c->kd, c->kk, c->red, c->xfer, c->d_status, c->d_sys, c->cta_bead, c->cta_spec,
                  c->cta_grid};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (SysHost& h : c->sys)
    for (int i = 0; i < TILD_MAX_COMPUTES; i++)
      if (h.sk[i]) cudaFree(h.sk[i]);
  tild_tables_free(c);
  for (auto& sl : c->snaps) {
    if (sl.dx) cudaFree(sl.dx);
    if (sl.drho) cudaFree(sl.drho);
    if (sl.captured) cudaEventDestroy(sl.captured);
    if (sl.done) cudaEventDestroy(sl.done);
  }
  if (c->snap_stream) cudaStreamDestroy(c->snap_stream);
  for (Bucket& b : c->buckets)
    if (b.planned) {
      cufftDestroy(b.fwd_packed ? b.c2c_fwd : b.r2c);
      cufftDestroy(b.packed ? b.c2c : b.c2r);
    }
  for (auto& ge : c->graphs) cudaGraphExecDestroy(ge.exec);
  c->graphs.clear();
  tild_sort_free(c);
  for (cudaStream_t a : c->aux) cudaStreamDestroy(a);
  for (cudaEvent_t e : c->ev_join) cudaEventDestroy(e);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->stream) cudaStreamDestroy(c->stream);
}

int validate(const tild_config* cfg, std::string& why) {
  char buf[256];
  if (cfg->dim != 2 && cfg->dim != 3) { why = "dim must be 2 or 3"; return TILD_ERR_BAD_INPUT; }
  if (cfg->pmeorder < 0 || cfg->pmeorder > 4) { why = "PMEORDER greater than 4 not supported!"; return TILD_ERR_BAD_INPUT; }
  if (cfg->ns <= 0) { why = "ns must be positive"; return TILD_ERR_BAD_INPUT; }
  if (cfg->ntypes < 1 || cfg->ntypes > TILD_MAX_TYPES) { why = "ntypes out of range (1..16)"; return TILD_ERR_BAD_INPUT; }
  for (int d = 0; d < cfg->dim; d++) {
    if (cfg->nx[d] < 1 || !(cfg->box[d] > 0.f)) { why = "grid sizes and box lengths must be positive"; return TILD_ERR_BAD_INPUT; }
    if (cfg->nx[d] < cfg->pmeorder + 1) { why = "grid smaller than the assignment stencil"; return TILD_ERR_BAD_INPUT; }
  }
  {
    long long m = 1;
    for (int d = 0; d < cfg->dim; d++) m *= cfg->nx[d];
    if (m >= (1ll << 31)) { why = "grids of 2^31 points or more are not supported"; return TILD_ERR_BAD_INPUT; }
  }
  if (cfg->n_styles < 0 || cfg->n_styles > TILD_MAX_STYLES) { why = "too many pair styles"; return TILD_ERR_BAD_INPUT; }
  for (int i = 0; i < cfg->n_styles; i++) {
    const tild_pair_style& s = cfg->styles[i];
    if (s.type1 < 0 || s.type2 < 0 || s.type1 >= cfg->ntypes || s.type2 >= cfg->ntypes) {
      snprintf(buf, sizeof buf, "Invalid particle type in pair style %d", i);
      why = buf;
      return TILD_ERR_BAD_INPUT;
    }
    if (s.style < TILD_STYLE_GAUSSIAN || s.style > TILD_STYLE_FIELDPHASE) { why = "unknown pair style"; return TILD_ERR_BAD_INPUT; }
    if (s.style == TILD_STYLE_FIELDPHASE) {
      if (s.phase != 0 && s.phase != 2 && s.phase != 3) { why = "fieldphase phase must be 0, 2 or 3 (BCC=1 is not implemented by gpu-tild)"; return TILD_ERR_BAD_INPUT; }
      if (s.dir < 0 || s.dir > 2 || (s.phase == 0 && s.dir >= cfg->dim)) { why = "fieldphase dir out of range"; return TILD_ERR_BAD_INPUT; }
    }
  }
  if (cfg->n_bond_types < 0 || cfg->n_bond_types > TILD_MAX_BOND_TYPES) { why = "too many bond types"; return TILD_ERR_BAD_INPUT; }
  if (cfg->n_integrators < 0 || cfg->n_integrators > TILD_MAX_INTEGRATORS) { why = "too many integrators"; return TILD_ERR_BAD_INPUT; }
  for (int k = 0; k < cfg->n_integrators; k++) {
    const tild_integrator& it = cfg->integrators[k];
    if (it.kind != TILD_INTEGRATOR_EM && it.kind != TILD_INTEGRATOR_GJF) { why = "is not a valid integrator!"; return TILD_ERR_BAD_INPUT; }
    if (it.group_type < -1 || it.group_type >= cfg->ntypes) { why = "integrator group type out of range"; return TILD_ERR_BAD_INPUT; }
  }
  // A bead whose integrator sequence has a GJF step after any other step would need its own
  // x_{n-1} buffer; the rotating two-buffer layout supports every other combination.
  for (int t = 0; t < cfg->ntypes; t++) {
    int seen = 0;
    for (int k = 0; k < cfg->n_integrators; k++) {
      const tild_integrator& it = cfg->integrators[k];
      if (it.group_type >= 0 && it.group_type != t) continue;
      if (it.kind == TILD_INTEGRATOR_GJF && seen) {
        why = "a GJF integrator preceded by another integrator on the same beads is not supported";
        return TILD_ERR_UNSUPPORTED;
      }
      seen++;
    }
  }
  if (cfg->rng != TILD_RNG_PHILOX && cfg->rng != TILD_RNG_XORWOW) { why = "unknown rng"; return TILD_ERR_BAD_INPUT; }
  return TILD_OK;
}

// Fixed-point scale of the shared-memory spread: 256 beads x the largest product of stencil
// weights (times the largest |q| on the charge channel) must stay below 2^31.
int spread_kbits(int P, int D, double gvol, double qmax) {
  double wmax = 0.0;
  for (int k = 0; k <= 1000; k++) {
    const double sx = -0.5 + k / 1000.0;
    double W[5];
    const double sx2 = sx * sx;
    double sx3, sx4;
    if (P == 0) { W[0] = 1; }
    else if (P == 1) { W[0] = 0.5 - sx; W[1] = 0.5 + sx; }
    else if (P == 2) { W[0] = 0.125 - 0.5 * sx + 0.5 * sx2; W[1] = 0.75 - sx2; W[2] = 0.125 + 0.5 * sx + 0.5 * sx2; }
    else if (P == 3) { sx3 = sx2 * sx; W[0] = (1 - 6 * sx + 12 * sx2 - 8 * sx3) / 48; W[1] = (23 - 30 * sx - 12 * sx2 + 24 * sx3) / 48;
                       W[2] = (23 + 30 * sx - 12 * sx2 - 24 * sx3) / 48; W[3] = (1 + 6 * sx + 12 * sx2 + 8 * sx3) / 48; }
    else { sx3 = sx2 * sx2; sx4 = sx2 * sx2; W[0] = (1 - 8 * sx + 24 * sx2 - 32 * sx3 + 16 * sx4) / 384;
           W[1] = (19 - 44 * sx + 24 * sx2 + 16 * sx3 - 16 * sx4) / 96; W[2] = (115 - 120 * sx2 + 48 * sx4) / 192;
           W[3] = (19 + 44 * sx + 24 * sx2 - 16 * sx3 - 16 * sx4) / 96; W[4] = (1 + 8 * sx + 24 * sx2 + 32 * sx3 + 16 * sx4) / 384; }
    for (int a = 0; a <= P; a++) wmax = std::max(wmax, std::fabs(W[a]));
  }
  const double bound = 256.0 * std::pow(wmax * 1.05, D) / gvol * std::max(qmax, 1.0);
  int k = 0;
  while (k < 31 && bound * std::ldexp(1.0, k + 1) < 2147483647.0) k++;
  return k;
}

}  // namespace

// Spreads the grid-shape buckets over the first `lanes` auxiliary streams (largest first, each to
// the least loaded stream) and binds their cuFFT plans to them; lanes = 0 keeps every transform on
// the main stream.
int tild_assign_lanes(tild_ctx* c, int lanes) {
  lanes = std::max(0, std::min(lanes, (int)c->aux.size()));
  std::vector<int> order(c->buckets.size());
  for (size_t k = 0; k < order.size(); k++) order[k] = (int)k;
  auto work = [&](int k) {
    const Bucket& b = c->buckets[k];
    return (long long)b.nx[0] * b.nx[1] * b.nx[2] * b.channels;
  };
  std::sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
  std::vector<long long> load(std::max(lanes, 1), 0);
  for (int bi : order) {
    Bucket& b = c->buckets[bi];
    if (lanes == 0) {
      b.lane = -1;
    } else {
      int best = 0;
      for (int k = 1; k < lanes; k++)
        if (load[k] < load[best]) best = k;
      b.lane = best;
      load[best] += work(bi);
    }
    if (!b.planned) continue;
    cudaStream_t bs = b.lane >= 0 ? c->aux[b.lane] : c->stream;
    if (tild_check_fft(c, cufftSetStream(b.fwd_packed ? b.c2c_fwd : b.r2c, bs), "plan stream") ||
        tild_check_fft(c, cufftSetStream(b.packed ? b.c2c : b.c2r, bs), "plan stream"))
      return 1;
  }
  c->lanes = lanes;
  return 0;
}

namespace {

// Geometry of a system from its configuration (initialize.cu:30-60).
void set_geometry(SysHost& h, const tild_config& cfg) {
  h.D = cfg.dim;
  h.T = cfg.ntypes;
  h.C = cfg.do_charges ? 1 : 0;
  h.ns = cfg.ns;
  h.p = cfg.pmeorder;
  h.nP = (h.D == 2) ? 3 : 6;
  Geom& g = h.g;
  g.M = 1;
  h.S = 1;
  float gv = 1.0f;
  for (int d = 0; d < 3; d++) {
    g.nx[d] = (d < h.D) ? cfg.nx[d] : 1;
    g.L[d] = (d < h.D) ? cfg.box[d] : 1.0f;
    g.Lh[d] = 0.5f * g.L[d];
    g.dx[d] = g.L[d] / (float)g.nx[d];
  }
  h.dV = 1.0;
  h.V = 1.0;
  for (int d = 0; d < h.D; d++) {
    gv *= g.dx[d];
    g.M *= g.nx[d];
    h.S *= (h.p + 1);
    h.dV *= (double)g.dx[d];
    h.V *= (double)g.L[d];
  }
  g.gvol = gv;
  g.nxh = g.nx[0] / 2 + 1;
  g.Mh = g.M / g.nx[0] * g.nxh;
}

// Physics part of system s's device descriptor (styles, integrators, masses, bonds) from h.cfg;
// the layout part (slots, offsets) and the step counter are left as they are.
void set_params(tild_ctx* c, int s) {
  SysHost& h = c->sys[s];
  const tild_config& cfg = h.cfg;
  SysDev& d = c->h_sys[s];
  h.fft_cfg.clear();
  int nfft = 0;
  for (int i = 0; i < cfg.n_styles; i++) {
    const tild_pair_style& ps = cfg.styles[i];
    if (ps.style == TILD_STYLE_FIELDPHASE) continue;
    d.sa[nfft] = ps.type1;
    d.sb[nfft] = ps.type2;
    d.sramp[nfft] = ps.ramp;
    d.sAi[nfft] = ps.prefactor;
    d.sAf[nfft] = ps.final_prefactor;
    d.suk0[nfft] = 1.0f;
    h.fft_cfg.push_back(i);
    nfft++;
  }
  for (int t = 0; t < TILD_MAX_TYPES; t++) h.type_integ_mask[t] = 0;
  for (int t = 0; t < h.T; t++) {
    int m = 0;
    for (int k = 0; k < cfg.n_integrators; k++)
      if (cfg.integrators[k].group_type < 0 || cfg.integrators[k].group_type == t) m |= 1 << k;
    h.type_integ_mask[t] = m;
  }
  d.g = h.g;
  d.T = h.T;
  d.C = h.C;
  d.nfft = nfft;
  d.ns = h.ns;
  d.max_steps = cfg.max_steps;
  d.seed = cfg.seed;
  d.delt = cfg.delt;
  d.noise_mag = cfg.noise_mag;
  d.n_integ = cfg.n_integrators;
  for (int k = 0; k < cfg.n_integrators; k++) d.integ_kind[k] = cfg.integrators[k].kind;
  for (int t = 0; t < h.T; t++) {
    d.type_mask[t] = h.type_integ_mask[t];
    d.mass[t] = cfg.mass[t];
    d.diff[t] = cfg.diff[t];
  }
  for (int b = 0; b < cfg.n_bond_types; b++) {
    d.bond_k[b] = cfg.bond_k[b];
    d.bond_req[b] = cfg.bond_req[b];
  }
  h.kbits = spread_kbits(h.p, h.D, h.g.gvol, 1.0);
  d.kbits = h.kbits;
}

int engine_create(const tild_config* cfgs, int nsys, int device, tild_ctx* c, const int32_t* capacity) {
  std::string why;
  for (int s = 0; s < nsys; s++) {
    int v = validate(&cfgs[s], why);
    if (v) {
      c->err = "system " + std::to_string(s) + ": " + why;
      return v;
    }
    if (cfgs[s].dim != cfgs[0].dim || cfgs[s].pmeorder != cfgs[0].pmeorder || cfgs[s].rng != cfgs[0].rng) {
      c->err = "systems of one batch must share dim, pmeorder and rng";
      return TILD_ERR_UNSUPPORTED;
    }
  }
  c->device = device;
  if (tild_check(c, cudaSetDevice(device), "cudaSetDevice")) return TILD_ERR_CUDA;
  if (tild_check(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) return TILD_ERR_CUDA;
  c->D = cfgs[0].dim;
  c->P = cfgs[0].pmeorder;
  c->rng = cfgs[0].rng;
  c->nsys = nsys;
  c->sys.resize(nsys);
  c->h_sys.assign(nsys, SysDev());
  memset(c->h_sys.data(), 0, sizeof(SysDev) * nsys);
  c->sort_interval = cfgs[0].sort_interval == 0 ? 16 : (cfgs[0].sort_interval < 0 ? 0 : cfgs[0].sort_interval);
  c->sort_brick = tild_brick_candidates(cfgs[0].dim == 2 ? 2 : 3)[0];
  c->steps_since_sort = c->sort_interval;
  c->spread_cap = 12288;
  // order <= 1 spreads by global atomics, which the gather absorbs at no cost; the order >= 2
  // shared box costs the gather its L1 share and barriers (both measured on the B200)
  c->spread_ahead = cfgs[0].pmeorder <= 1 ? 1 : 0;
  long long slots = 0, beads = 0, utab = 0, virk = 0, ctab = 0, kd = 0, fr = 0;
  // buckets by grid shape (order of first appearance)
  for (int s = 0; s < nsys; s++) {
    const tild_config& cfg = cfgs[s];
    SysHost& h = c->sys[s];
    h.cfg = cfg;
    set_geometry(h, cfg);
    const Geom& g = h.g;
    h.cap = capacity ? std::max(h.ns, (int)capacity[s]) : h.ns;
    h.ns_pad = (h.cap + kTile - 1) / kTile * kTile;
    for (int i = 0; i < cfg.n_styles; i++)
      if (cfg.styles[i].style == TILD_STYLE_FIELDPHASE) {
        FieldK f;
        f.sys = s;
        f.a = cfg.styles[i].type1;
        f.b = cfg.styles[i].type2;
        f.cfg_index = i;
        f.fr0 = fr;
        fr += (long long)h.D * g.M;
        c->fields.push_back(f);
      }
    set_params(c, s);
    const int nfft = (int)h.fft_cfg.size();
    h.utab0 = utab;
    utab += (long long)nfft * g.Mh;
    h.virk0 = virk;
    virk += (long long)nfft * h.nP * g.Mh;
    h.ctab0 = ctab;
    ctab += (long long)h.C * g.Mh;
    h.kd0 = kd;
    kd += g.nx[0] + g.nx[1] + g.nx[2];
    c->maxT = std::max(c->maxT, h.T);
    c->any_charges |= h.C != 0;
    int bi = -1;
    for (size_t k = 0; k < c->buckets.size(); k++)
      if (c->buckets[k].nx[0] == g.nx[0] && c->buckets[k].nx[1] == g.nx[1] && c->buckets[k].nx[2] == g.nx[2]) bi = (int)k;
    if (bi < 0) {
      Bucket b;
      for (int q = 0; q < 3; q++) b.nx[q] = g.nx[q];
      c->buckets.push_back(b);
      bi = (int)c->buckets.size() - 1;
    }
    c->buckets[bi].systems.push_back(s);
    h.bucket = bi;
    // layout part of the device descriptor (slots are placed below, shape by shape)
    SysDev& d = c->h_sys[s];
    d.ns_pad = h.ns_pad;
    d.active = 1;
    d.utab0 = h.utab0;
    d.ctab0 = h.ctab0;
    d.kd0 = h.kd0;
    d.step = 0;
    d.stop_at = -1;
  }
  // channel layout: bucket by bucket so each bucket is one batched transform
  long long grid = 0, spec = 0;
  long long g4tot = 0;
  int rank = 0;
  for (Bucket& b : c->buckets) {
    b.grid0 = grid;
    b.spec0 = spec;
    b.channels = 0;
    for (int s : b.systems) {
      SysHost& h = c->sys[s];
      // slots shape by shape too, so that a shape's beads are one range of particle blocks
      h.slot0 = (int)slots;
      h.bead0 = (int)beads;
      slots += h.ns_pad;
      beads += h.cap;
      c->h_sys[s].slot0 = h.slot0;
      c->h_sys[s].bead0 = h.bead0;
      c->h_sys[s].slot_rank = rank++;
      h.grid0 = grid;
      h.spec0 = spec;
      h.Mb = tild_field_stride(h.g, h.D);
      h.g4_0 = g4tot;
      g4tot += (long long)(h.T + h.C) * h.Mb;
      c->h_sys[s].grid0 = grid;
      c->h_sys[s].spec0 = spec;
      c->h_sys[s].g4_0 = h.g4_0;
      c->h_sys[s].Mb = h.Mb;
      grid += (long long)(h.T + h.C) * h.g.M;
      spec += (long long)(h.T + h.C) * h.g.Mh;
      b.channels += h.T + h.C;
    }
    // the inverse transforms pair channels when every system has an even number of them and none
    // has a fieldphase style (those add to the planar fields between transform and interleave);
    // each system's pair spectra follow one another, transformed in place
    b.packed = true;
    for (int s : b.systems) {
      const SysHost& h = c->sys[s];
      if ((h.T + h.C) % 2) b.packed = false;
      for (const FieldK& f : c->fields) b.packed = b.packed && f.sys != s;
    }
    // the forward transforms pair them the same way when the bucket's densities start on a complex
    // boundary (they are read as complex pairs); the pair spectra follow one another in rhok
    b.fwd_packed = b.packed && b.grid0 % 2 == 0;
    long long pairs = 0;
    for (int s : b.systems) {
      const SysHost& h = c->sys[s];
      c->h_sys[s].inv_packed = b.packed ? 1 : 0;
      c->h_sys[s].gkp0 = b.packed ? b.spec0 * c->D + pairs * c->D * h.g.M : 0;
      c->h_sys[s].fwd_packed = b.fwd_packed ? 1 : 0;
      c->h_sys[s].rkp0 = b.fwd_packed ? b.spec0 + pairs * h.g.M : 0;
      pairs += (h.T + h.C) / 2;
    }
  }
  c->grid_total = grid;
  c->spec_total = spec;
  c->g4_total = g4tot;
  c->nslots = (int)slots;
  c->nbeads = (int)beads;
  // CTA -> system lookup tables (grid and spectrum tables carry each system's first block after them)
  std::vector<int> tb, tspec, tgrid, bspec(nsys), bgrid(nsys);
  // particle, spectrum and grid blocks in grid-shape order, so each shape's blocks form one range
  for (Bucket& b : c->buckets) {
    b.cta_bead0 = (int)tb.size();
    b.cta_spec0 = (int)tspec.size();
    b.cta_grid0 = (int)tgrid.size();
    for (int s : b.systems) {
      for (int k = 0; k < c->sys[s].ns_pad / kTile; k++) tb.push_back(s);
      bspec[s] = (int)tspec.size();
      for (long long k = 0; k < (c->sys[s].g.Mh + 255) / 256; k++) tspec.push_back(s);
      bgrid[s] = (int)tgrid.size();
      for (long long k = 0; k < (c->sys[s].g.M + 255) / 256; k++) tgrid.push_back(s);
    }
    b.n_cta_bead = (int)tb.size() - b.cta_bead0;
    b.n_cta_spec = (int)tspec.size() - b.cta_spec0;
    b.n_cta_grid = (int)tgrid.size() - b.cta_grid0;
  }
  c->n_cta_bead = (int)tb.size();
  c->n_cta_spec = (int)tspec.size();
  c->n_cta_grid = (int)tgrid.size();
  tspec.insert(tspec.end(), bspec.begin(), bspec.end());
  tgrid.insert(tgrid.end(), bgrid.begin(), bgrid.end());
  int maxns = 1;
  for (const SysHost& h : c->sys) maxns = std::max(maxns, h.cap);
  const size_t NS = c->nslots;
  int rc = TILD_OK;
  rc = rc ? rc : dalloc(c, &c->pos[0], NS, "positions");
  rc = rc ? rc : dalloc(c, &c->pos[1], NS, "positions");
  rc = rc ? rc : dalloc(c, &c->noise, NS * 3, "noise");
  rc = rc ? rc : dalloc(c, &c->bead_id, NS, "bead ids");
  rc = rc ? rc : dalloc(c, &c->slot_of, (size_t)c->nbeads, "slots");
  rc = rc ? rc : dalloc(c, &c->bond_nbr, NS * 3, "bonds");
  rc = rc ? rc : dalloc(c, &c->bond_info, NS, "bonds");
  rc = rc ? rc : dalloc(c, &c->types_dev, (size_t)c->nbeads, "types");
  if (c->any_charges) rc = rc ? rc : dalloc(c, &c->charge, NS, "charges");
  rc = rc ? rc : dalloc(c, &c->rho, (size_t)grid, "densities");
  rc = rc ? rc : dalloc(c, &c->rho_fx, (size_t)grid, "density accumulator");
  rc = rc ? rc : dalloc(c, &c->rhok, (size_t)spec, "density spectra");
  rc = rc ? rc : dalloc(c, &c->gk, (size_t)spec * c->D, "force spectra");
  bool any_c2r = false;  // planar force fields are only needed by buckets whose inverse is C2R
  for (const Bucket& b : c->buckets) any_c2r = any_c2r || !b.packed;
  rc = rc ? rc : dalloc(c, &c->gfield, any_c2r ? (size_t)grid * c->D : 1, "force fields");
  rc = rc ? rc : dalloc(c, &c->g4, (size_t)c->g4_total, "interleaved force fields");
  rc = rc ? rc : dalloc(c, &c->utab, (size_t)utab, "multiplier tables");
  rc = rc ? rc : dalloc(c, &c->virk, (size_t)virk, "virial tables");
  if (ctab) rc = rc ? rc : dalloc(c, &c->ctab, (size_t)ctab, "charge table");
  if (fr) rc = rc ? rc : dalloc(c, &c->frfield, (size_t)fr, "fieldphase fields");
  rc = rc ? rc : dalloc(c, &c->kd, (size_t)kd, "k vectors");
  rc = rc ? rc : dalloc(c, &c->kk, (size_t)kd, "k vectors");
  rc = rc ? rc : dalloc(c, &c->xfer, (size_t)maxns * 3, "transfer buffer");
  rc = rc ? rc : dalloc(c, &c->d_status, 2, "status");  // [0] status word, [1] input check flag
  rc = rc ? rc : dalloc(c, &c->d_sys, (size_t)nsys, "system descriptors");
  rc = rc ? rc : dalloc(c, &c->cta_bead, tb.size(), "lookup");
  rc = rc ? rc : dalloc(c, &c->cta_spec, tspec.size(), "lookup");
  rc = rc ? rc : dalloc(c, &c->cta_grid, tgrid.size(), "lookup");
  if (c->rng == TILD_RNG_XORWOW) rc = rc ? rc : dalloc(c, &c->xorwow, NS, "xorwow states");
  if (rc) return rc;
  cudaStream_t st = c->stream;
  cudaMemsetAsync(c->d_status, 0, 2 * sizeof(int), st);
  cudaMemsetAsync(c->rho_fx, 0, sizeof(unsigned long long) * grid, st);
  cudaMemsetAsync(c->noise, 0, sizeof(float) * NS * 3, st);
  cudaMemsetAsync(c->bond_nbr, 0, sizeof(int) * NS * 3, st);
  cudaMemsetAsync(c->bond_info, 0, sizeof(int) * NS, st);
  cudaMemsetAsync(c->bead_id, 0xff, sizeof(int) * NS, st);
  if (c->charge) cudaMemsetAsync(c->charge, 0, sizeof(float) * NS, st);
  k_fill_padding<<<nblk(NS, 256), 256, 0, st>>>(c->pos[0], c->pos[1], (int)NS);
  c->launches++;
  cudaMemcpyAsync(c->cta_bead, tb.data(), tb.size() * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->cta_spec, tspec.data(), tspec.size() * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->cta_grid, tgrid.data(), tgrid.size() * 4, cudaMemcpyHostToDevice, st);
  if (tild_check(c, cudaStreamSynchronize(st), "init")) return TILD_ERR_CUDA;
  // batched cuFFT plans, one pair per grid shape; with several shapes each plan runs on one of
  // up to 8 auxiliary streams so transforms of different shapes overlap
  if (c->buckets.size() > 1) {
    const int naux = (int)std::min<size_t>(8, c->buckets.size());
    c->aux.resize(naux);
    c->ev_join.resize(naux);
    for (int k = 0; k < naux; k++) {
      if (tild_check(c, cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking), "aux stream") ||
          tild_check(c, cudaEventCreateWithFlags(&c->ev_join[k], cudaEventDisableTiming), "aux event"))
        return TILD_ERR_CUDA;
    }
    if (tild_check(c, cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming), "fork event")) return TILD_ERR_CUDA;
  }
  for (Bucket& b : c->buckets) {
    int n[3];
    if (c->D == 3) { n[0] = b.nx[2]; n[1] = b.nx[1]; n[2] = b.nx[0]; }
    else { n[0] = b.nx[1]; n[1] = b.nx[0]; }
    const cufftResult pf = b.fwd_packed
        ? cufftPlanMany(&b.c2c_fwd, c->D, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, b.channels / 2)
        : cufftPlanMany(&b.r2c, c->D, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, b.channels);
    if (tild_check_fft(c, pf, b.fwd_packed ? "plan C2C forward" : "plan R2C")) return TILD_ERR_CUDA;
    const cufftResult pi = b.packed
        ? cufftPlanMany(&b.c2c, c->D, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, b.channels / 2 * c->D)
        : cufftPlanMany(&b.c2r, c->D, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, b.channels * c->D);
    if (tild_check_fft(c, pi, b.packed ? "plan C2C" : "plan C2R")) {
      cufftDestroy(b.fwd_packed ? b.c2c_fwd : b.r2c);
      return TILD_ERR_CUDA;
    }
    b.planned = true;
  }
  if (tild_assign_lanes(c, (int)c->aux.size())) return TILD_ERR_CUDA;
  for (int s = 0; s < nsys && !rc; s++) rc = tild_build_tables(c, s);
  if (rc) return rc;
  if (c->sort_interval > 0) {
    rc = tild_sort_alloc(c);
    if (rc) return rc;
  }
  return tild_upload_sys(c);
}

int check_sys(tild_ctx* c, int s) {
  if (!c || s < 0 || s >= c->nsys) return TILD_ERR_BAD_INPUT;
  return TILD_OK;
}

int sys_set_topology(tild_ctx* c, int s, const int32_t* types, const float* charges, const int32_t* n_bonds,
                     const int32_t* bonded_to, const int32_t* bond_type) {
  if (check_sys(c, s) || !types) return TILD_ERR_BAD_INPUT;
  SysHost& h = c->sys[s];
  if (h.C && !charges) return set_err(c, TILD_ERR_BAD_INPUT, "charges required when do_charges is set");
  cudaSetDevice(c->device);
  if (tild_drop_ahead(c)) return TILD_ERR_CUDA;
  const int ns = h.ns, np = h.ns_pad;
  std::vector<int> nbr(3 * (size_t)np, 0), info(np, 0), bid(np, -1), slot_of(ns);
  std::vector<float> q;
  if (c->charge) q.assign(np, 0.f);
  double qmax = 1.0;
  for (int b = 0; b < ns; b++) {
    if (types[b] < 0 || types[b] >= h.T) return set_err(c, TILD_ERR_BAD_INPUT, "bead type out of range");
    int nb = n_bonds ? n_bonds[b] : 0;
    if (nb < 0 || nb > TILD_MAX_BONDS) return set_err(c, TILD_ERR_BAD_INPUT, "more than MAX_BONDS (3) bonds on a bead");
    int in = nb;
    for (int k = 0; k < nb; k++) {
      const int j = bonded_to[3 * (size_t)b + k], bt = bond_type[3 * (size_t)b + k];
      if (j < 0 || j >= ns) return set_err(c, TILD_ERR_BAD_INPUT, "bond partner out of range");
      if (bt < 0 || bt >= h.cfg.n_bond_types) return set_err(c, TILD_ERR_BAD_INPUT, "bond type out of range");
      nbr[3 * (size_t)b + k] = h.slot0 + j;
      in |= bt << (8 + 8 * k);
    }
    info[b] = in;
    bid[b] = b;
    slot_of[b] = h.slot0 + b;
    if (h.C) {
      q[b] = charges[b];
      qmax = std::max(qmax, (double)std::fabs(charges[b]));
    }
  }
  cudaStream_t st = c->stream;
  if (tild_check(c, cudaMemcpyAsync(c->bond_nbr + 3 * (size_t)h.slot0, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, st), "bonds") ||
      tild_check(c, cudaMemcpyAsync(c->bond_info + h.slot0, info.data(), info.size() * 4, cudaMemcpyHostToDevice, st), "bonds") ||
      tild_check(c, cudaMemcpyAsync(c->bead_id + h.slot0, bid.data(), bid.size() * 4, cudaMemcpyHostToDevice, st), "ids") ||
      tild_check(c, cudaMemcpyAsync(c->slot_of + h.bead0, slot_of.data(), slot_of.size() * 4, cudaMemcpyHostToDevice, st), "slots") ||
      tild_check(c, cudaMemcpyAsync(c->types_dev + h.bead0, types, (size_t)ns * 4, cudaMemcpyHostToDevice, st), "types") ||
      (c->charge && tild_check(c, cudaMemcpyAsync(c->charge + h.slot0, q.data(), (size_t)np * 4, cudaMemcpyHostToDevice, st), "charges")))
    return TILD_ERR_CUDA;
  k_fill_padding<<<nblk(np, 256), 256, 0, st>>>(c->pos[0] + h.slot0, c->pos[1] + h.slot0, np);
  c->launches++;
  if (tild_check(c, cudaStreamSynchronize(st), "sync topology")) return TILD_ERR_CUDA;
  h.kbits = spread_kbits(h.p, h.D, h.g.gvol, qmax);
  c->h_sys[s].kbits = h.kbits;
  h.topo_set = true;
  h.state_set = false;
  h.have_forces = false;
  return tild_upload_sys(c);
}

int sys_set_state(tild_ctx* c, int s, const float* x, const float* xo, const float* prev_noise) {
  if (check_sys(c, s) || !x) return TILD_ERR_BAD_INPUT;
  SysHost& h = c->sys[s];
  if (!h.topo_set) return set_err(c, TILD_ERR_STATE, "tild_set_topology must come before tild_set_state");
  cudaSetDevice(c->device);
  const size_t n = (size_t)h.ns * h.D;
  const unsigned nb = nblk(h.ns, 256);
  cudaStream_t st = c->stream;
  const int* so = c->slot_of + h.bead0;
  const int* ty = c->types_dev + h.bead0;
  if (tild_check(c, cudaMemcpyAsync(c->xfer, x, n * 4, cudaMemcpyHostToDevice, st), "upload x")) return TILD_ERR_CUDA;
  // the positions are checked on the device before anything of the current state changes
  {
    int bad = 0;
    if (tild_check(c, cudaMemsetAsync(c->d_status + 1, 0, sizeof(int), st), "clear check flag")) return TILD_ERR_CUDA;
    k_check_finite<<<std::min<unsigned>(nblk((long long)n, 256), 1184), 256, 0, st>>>(c->xfer, (long long)n,
                                                                                        c->d_status + 1);
    c->launches++;
    if (tild_check(c, cudaMemcpyAsync(&bad, c->d_status + 1, sizeof(int), cudaMemcpyDeviceToHost, st), "check flag") ||
        tild_check(c, cudaStreamSynchronize(st), "sync check"))
      return TILD_ERR_CUDA;
    if (bad) return set_err(c, TILD_ERR_NAN, "non-finite position in tild_set_state");
  }
  if (tild_drop_ahead(c)) return TILD_ERR_CUDA;
  k_pack_pos<<<nb, 256, 0, st>>>(c->xfer, ty, so, h.ns, h.D, c->pos[c->cur]);
  // x_{n-1}: xo when given, else x (send_3n_to_device copies x into xo, device_comm_utils.cu:15-16)
  if (xo && tild_check(c, cudaMemcpyAsync(c->xfer, xo, n * 4, cudaMemcpyHostToDevice, st), "upload xo"))
    return TILD_ERR_CUDA;
  k_pack_pos<<<nb, 256, 0, st>>>(c->xfer, ty, so, h.ns, h.D, c->pos[c->cur ^ 1]);
  if (prev_noise && tild_check(c, cudaMemcpyAsync(c->xfer, prev_noise, n * 4, cudaMemcpyHostToDevice, st), "upload noise"))
    return TILD_ERR_CUDA;
  k_pack_noise<<<nb, 256, 0, st>>>(prev_noise ? c->xfer : nullptr, so, h.ns, h.D, c->noise);
  c->launches += 3;
  if (c->xorwow) {
    k_init_xorwow<<<nblk(h.ns_pad, 256), 256, 0, st>>>(c->xorwow + h.slot0, c->bead_id + h.slot0, h.ns_pad,
                                                        (unsigned int)h.cfg.seed);
    c->launches++;
  }
  if (tild_check(c, cudaStreamSynchronize(st), "set state")) return TILD_ERR_CUDA;
  c->steps_since_sort = c->sort_interval;  // sort before the next step
  h.state_set = true;
  h.have_forces = false;
  return TILD_OK;
}

int sys_get_state(tild_ctx* c, int s, float* x, float* xo, float* prev_noise) {
  if (check_sys(c, s)) return TILD_ERR_BAD_INPUT;
  SysHost& h = c->sys[s];
  if (!h.state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  const size_t n = (size_t)h.ns * h.D;
  const unsigned nb = nblk(h.ns_pad, 256);
  float* outs[3] = {x, xo, prev_noise};
  for (int k = 0; k < 3; k++) {
    if (!outs[k]) continue;
    if (k < 2)
      k_unpack_pos<<<nb, 256, 0, c->stream>>>(c->pos[k == 0 ? c->cur : c->cur ^ 1] + h.slot0, c->bead_id + h.slot0,
                                               h.ns_pad, h.D, c->xfer);
    else
      k_unpack_noise<<<nb, 256, 0, c->stream>>>(c->noise + 3 * (size_t)h.slot0, c->bead_id + h.slot0, h.ns_pad, h.D,
                                                 c->xfer);
    c->launches++;
    if (tild_check(c, cudaMemcpyAsync(outs[k], c->xfer, n * 4, cudaMemcpyDeviceToHost, c->stream), "download") ||
        tild_check(c, cudaStreamSynchronize(c->stream), "sync download"))
      return TILD_ERR_CUDA;
  }
  return TILD_OK;
}

bool all_ready(tild_ctx* c) {
  for (const SysHost& h : c->sys)
    if (h.active && !h.state_set) return false;
  return true;
}

// Host bookkeeping of `n` integrating steps that ran inside a graph replay (the device side,
// including step counters and buffer rotations, is in the graph).
void account_replayed_steps(tild_ctx* c, int n, long long launches, int nsorts) {
  for (int s = 0; s < c->nsys; s++) {
    SysHost& h = c->sys[s];
    if (!h.active) continue;
    h.step += n;
    c->h_sys[s].step = h.step;
    h.forces_step = h.step;
    h.have_forces = true;
  }
  c->launches += launches;
  c->sorts += nsorts;
}

constexpr int kMinGraphSteps = 8;  // shorter runs launch directly

// n integrating steps as CUDA graphs.  Whole periods of graph_len steps (two sort periods, so
// every buffer rotation and sort trade returns to its starting configuration) start with a sort;
// a remainder of at least kMinGraphSteps steps (or a run that starts between sorts) is a graph
// of its own length.  A graph is captured once per starting configuration (buffers, rotation,
// sort phase, spread-ahead state, transformed grid shapes, length) and replayed afterwards; a
// replay moves the host mirrors to the configuration the capture ended in.  Shorter remainders
// run as direct launches.
int run_steps(tild_ctx* c, int n) {
  const int len = c->sort_interval > 0 ? 2 * c->sort_interval : c->graph_len;
  while (n > 0) {
    const bool aligned = c->sort_interval <= 0 || c->steps_since_sort >= c->sort_interval;
    int L = 0;
    if (c->use_graphs && !c->profiling) {
      if (n >= len && aligned) L = len;
      else if (n >= kMinGraphSteps) L = std::min(n, len);
    }
    if (L == 0) {
      int rc = tild_run_forces(c, true, nullptr, -1);
      if (rc) return rc;
      n -= 1;
      continue;
    }
    if (L == len && aligned) c->steps_since_sort = c->sort_interval;  // a whole period starts with a sort
    const void* p0 = c->pos[0];
    const int cur = c->cur;
    const int64_t sss0 = c->steps_since_sort;
    const std::vector<char> on = tild_buckets_on(c);
    const bool ahead = c->rho_ahead;  // whether the graph's first step spreads
    const tild_ctx::GraphEntry* found = nullptr;
    for (const auto& ge : c->graphs)
      if (ge.p0 == p0 && ge.cur == cur && ge.buckets_on == on && ge.ahead == ahead && ge.len == L && ge.sss0 == sss0)
        found = &ge;
    if (found) {
      const tild_ctx::GraphEntry ge = *found;
      if (tild_check(c, cudaGraphLaunch(ge.exec, c->stream), "graph launch")) return TILD_ERR_CUDA;
      c->cur = ge.cur_end;
      for (int k = 0; k < (ge.nsorts & 1); k++) tild_sort_swap_buffers(c);
      c->steps_since_sort = ge.sss_end;
      c->rho_ahead = ge.ahead_end;
      account_replayed_steps(c, L, ge.launches, ge.nsorts);
      n -= L;
      continue;
    }
    // capture: the host code runs the steps' launches into the graph and leaves every host
    // mirror of the buffers at the configuration after them; the step counters are put back
    // and advance when the graph runs
    const long long l0 = c->launches;
    std::vector<SysHost> saved_hosts;
    for (const SysHost& h : c->sys) saved_hosts.push_back(h);
    const auto saved_hsys = c->h_sys;
    const long long saved_sorts = c->sorts;
    if (tild_check(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed), "begin capture"))
      return TILD_ERR_CUDA;
    int rc = TILD_OK;
    for (int k = 0; k < L && !rc; k++) rc = tild_run_forces(c, true, nullptr, -1);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (tild_check(c, e, "end capture")) return TILD_ERR_CUDA;
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (tild_check(c, ei, "instantiate graph")) return TILD_ERR_CUDA;
    const long long glaunches = c->launches - l0;
    const int nsorts = (int)(c->sorts - saved_sorts);
    for (int s = 0; s < c->nsys; s++) {
      c->sys[s].step = saved_hosts[s].step;
      c->sys[s].forces_step = saved_hosts[s].forces_step;
      c->sys[s].have_forces = saved_hosts[s].have_forces;
    }
    c->h_sys = saved_hsys;
    c->sorts = saved_sorts;
    c->launches = l0;
    if (c->graphs.size() >= 8) {  // keep the eight most recent configurations
      cudaGraphExecDestroy(c->graphs.front().exec);
      c->graphs.erase(c->graphs.begin());
    }
    c->graphs.push_back({exec, p0, cur, on, ahead, c->rho_ahead, L, sss0, c->steps_since_sort, c->cur, nsorts, glaunches});
    c->graph_launches_per_step = glaunches / L;
    if (tild_check(c, cudaGraphLaunch(exec, c->stream), "graph launch")) return TILD_ERR_CUDA;
    account_replayed_steps(c, L, glaunches, nsorts);
    n -= L;
  }
  return TILD_OK;
}

// Systems with a stop step leave the active set on the device (k_advance_steps): bring their
// step counters and activity back into the host mirrors after every stepping call.
int refresh_from_device(tild_ctx* c) {
  if (!c->any_stop) return TILD_OK;
  std::vector<SysDev> dev(c->nsys);
  if (tild_check(c, cudaMemcpyAsync(dev.data(), c->d_sys, sizeof(SysDev) * c->nsys, cudaMemcpyDeviceToHost, c->stream),
                 "download descriptors") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync descriptors"))
    return TILD_ERR_CUDA;
  for (int s = 0; s < c->nsys; s++) {
    SysHost& h = c->sys[s];
    h.step = dev[s].step;
    c->h_sys[s].step = dev[s].step;
    h.active = h.active && dev[s].active;
    c->h_sys[s].active = h.active ? 1 : 0;
  }
  return TILD_OK;
}

int engine_step(tild_ctx* c, int nsteps) {
  if (!all_ready(c)) return set_err(c, TILD_ERR_STATE, "every active system needs tild_set_state before stepping");
  cudaSetDevice(c->device);
  int rc = run_steps(c, nsteps);
  if (!rc) rc = refresh_from_device(c);
  if (rc) return rc;
  return tild_poll_status(c);
}

int sys_forces(tild_ctx* c, int s, float* f) {
  if (check_sys(c, s)) return TILD_ERR_BAD_INPUT;
  if (!all_ready(c)) return set_err(c, TILD_ERR_STATE, "tild_set_state must come before tild_forces");
  cudaSetDevice(c->device);
  int rc = tild_run_forces(c, false, f ? c->xfer : nullptr, s);
  if (rc) return rc;
  rc = tild_poll_status(c);
  if (rc) return rc;
  if (f) {
    const SysHost& h = c->sys[s];
    if (tild_check(c, cudaMemcpyAsync(f, c->xfer, (size_t)h.ns * h.D * 4, cudaMemcpyDeviceToHost, c->stream), "download f") ||
        tild_check(c, cudaStreamSynchronize(c->stream), "sync f"))
      return TILD_ERR_CUDA;
  }
  return TILD_OK;
}

int sys_observables(tild_ctx* c, int s, tild_obs* o) {
  if (check_sys(c, s) || !o) return TILD_ERR_BAD_INPUT;
  if (!c->sys[s].state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  if (!c->sys[s].have_forces) {
    int rc = tild_run_forces(c, false, nullptr, -1);
    if (rc) return rc;
  }
  int rc = tild_obs_compute(c, s, o);
  if (rc) return rc;
  if (!std::isfinite(o->upe)) return set_err(c, TILD_ERR_NAN, "non-finite energy");
  return tild_poll_status(c);
}

int sys_density(tild_ctx* c, int s, float* rho) {
  if (check_sys(c, s) || !rho) return TILD_ERR_BAD_INPUT;
  const SysHost& h = c->sys[s];
  if (!h.have_forces) return set_err(c, TILD_ERR_STATE, "no force evaluation yet");
  cudaSetDevice(c->device);
  const float* src = c->rho + h.grid0;
  if (c->h_sys[s].fwd_packed) {  // paired layout: planar channels staged in the force-field scratch first
    float* planar = reinterpret_cast<float*>(c->gk) + h.grid0;
    if (tild_density_planar(c, s, planar, c->stream)) return TILD_ERR_CUDA;
    src = planar;
  }
  if (tild_check(c, cudaMemcpyAsync(rho, src, sizeof(float) * (size_t)(h.T + h.C) * h.g.M, cudaMemcpyDeviceToHost, c->stream), "download rho") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync rho"))
    return TILD_ERR_CUDA;
  return TILD_OK;
}

int sys_set_step(tild_ctx* c, int s, int64_t step) {
  if (check_sys(c, s) || step < 0) return TILD_ERR_BAD_INPUT;
  c->sys[s].step = step;
  c->h_sys[s].step = step;
  return tild_upload_sys(c);
}

int engine_time(tild_ctx* c, int nsteps, double* ms) {
  if (!c || !ms || nsteps < 0) return TILD_ERR_BAD_INPUT;
  if (!all_ready(c)) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  int rc = run_steps(c, nsteps);
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) rc = refresh_from_device(c);
  return rc ? rc : tild_poll_status(c);
}

// Replaces the system of slot s by another of the same grid shape and channel layout.
int sys_load(tild_ctx* c, int s, const tild_config* cfg) {
  if (check_sys(c, s) || !cfg) return TILD_ERR_BAD_INPUT;
  std::string why;
  const int v = validate(cfg, why);
  if (v) return set_err(c, v, why.c_str());
  SysHost& h = c->sys[s];
  if (cfg->dim != c->D || cfg->pmeorder != c->P || cfg->rng != c->rng)
    return set_err(c, TILD_ERR_UNSUPPORTED, "dim, pmeorder and rng must match the batch");
  for (int d = 0; d < 3; d++)
    if ((d < c->D ? cfg->nx[d] : 1) != h.g.nx[d]) return set_err(c, TILD_ERR_UNSUPPORTED, "grid shape differs from the slot's");
  if (cfg->ntypes != h.T || (cfg->do_charges ? 1 : 0) != h.C)
    return set_err(c, TILD_ERR_UNSUPPORTED, "ntypes and do_charges must match the slot");
  if (cfg->ns > h.cap) return set_err(c, TILD_ERR_UNSUPPORTED, "more beads than the slot holds");
  int nfft = 0, nfield = 0, nfield_slot = 0;
  for (int i = 0; i < cfg->n_styles; i++) (cfg->styles[i].style == TILD_STYLE_FIELDPHASE ? nfield : nfft)++;
  for (const FieldK& fk : c->fields) nfield_slot += fk.sys == s;
  if (nfft != (int)h.fft_cfg.size() || nfield != nfield_slot)
    return set_err(c, TILD_ERR_UNSUPPORTED, "the slot's number of FFT pair styles and of fieldphases must match");
  cudaSetDevice(c->device);
  if (tild_drop_ahead(c)) return TILD_ERR_CUDA;
  if (tild_check(c, cudaStreamSynchronize(c->stream), "sync before load")) return TILD_ERR_CUDA;
  h.cfg = *cfg;
  set_geometry(h, *cfg);
  set_params(c, s);
  bool fields_moved = false;
  for (int i = 0, k = 0; i < cfg->n_styles; i++) {
    if (cfg->styles[i].style != TILD_STYLE_FIELDPHASE) continue;
    while (c->fields[k].sys != s) k++;
    FieldK& fk = c->fields[k++];
    fields_moved |= fk.a != cfg->styles[i].type1 || fk.b != cfg->styles[i].type2;
    fk.a = cfg->styles[i].type1;
    fk.b = cfg->styles[i].type2;
    fk.cfg_index = i;
  }
  if (fields_moved) {  // the captured step graphs carry the fieldphase types as launch arguments
    for (auto& ge : c->graphs) cudaGraphExecDestroy(ge.exec);
    c->graphs.clear();
  }
  SysDev& d = c->h_sys[s];
  d.step = 0;
  d.stop_at = -1;
  h.step = 0;
  h.forces_step = 0;
  h.active = false;
  h.topo_set = h.state_set = h.have_forces = false;
  for (int k = 0; k < TILD_MAX_COMPUTES; k++) {
    if (h.sk[k] && tild_check(c, cudaMemsetAsync(h.sk[k], 0, sizeof(double2) * h.g.Mh, c->stream), "clear sk"))
      return TILD_ERR_CUDA;
    h.sk_calls[k] = 0;
  }
  const int rc = tild_build_tables(c, s);
  if (rc) return rc;
  return tild_upload_sys(c);
}

int sys_sk_accumulate(tild_ctx* c, int s, int slot, int type) {
  if (check_sys(c, s) || slot < 0 || slot >= TILD_MAX_COMPUTES || type < 0 || type >= c->sys[s].T)
    return TILD_ERR_BAD_INPUT;
  if (!c->sys[s].have_forces) return set_err(c, TILD_ERR_STATE, "no force evaluation yet");
  cudaSetDevice(c->device);
  return tild_sk_acc_run(c, s, slot, type);
}

int sys_sk_get(tild_ctx* c, int s, int slot, double* sk, int32_t* ncalls) {
  if (check_sys(c, s) || slot < 0 || slot >= TILD_MAX_COMPUTES) return TILD_ERR_BAD_INPUT;
  cudaSetDevice(c->device);
  const SysHost& h = c->sys[s];
  const int n = h.sk[slot] ? h.sk_calls[slot] : 0;
  if (ncalls) *ncalls = n;
  if (!sk) return TILD_OK;
  const Geom& g = h.g;
  if (n == 0) {
    memset(sk, 0, sizeof(double) * 2 * (size_t)g.M);
    return TILD_OK;
  }
  std::vector<double> hb(2 * (size_t)g.Mh);
  if (tild_check(c, cudaMemcpyAsync(hb.data(), h.sk[slot], sizeof(double) * hb.size(), cudaMemcpyDeviceToHost, c->stream), "download sk") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync sk"))
    return TILD_ERR_CUDA;
  // expand the half spectrum: A(-k) = conj(A(k)) for A = rho_k * rho_k of a real density
  const int N0 = g.nx[0], N1 = g.nx[1], N2 = g.nx[2];
  for (int z = 0; z < N2; z++)
    for (int y = 0; y < N1; y++)
      for (int x = 0; x < N0; x++) {
        const size_t id = (size_t)x + (size_t)N0 * (y + (size_t)N1 * z);
        double re, im;
        if (x < g.nxh) {
          const size_t h2 = (size_t)x + (size_t)g.nxh * (y + (size_t)N1 * z);
          re = hb[2 * h2];
          im = hb[2 * h2 + 1];
        } else {
          const int xm = N0 - x, ym = (N1 - y) % N1, zm = (N2 - z) % N2;
          const size_t h2 = (size_t)xm + (size_t)g.nxh * (ym + (size_t)N1 * zm);
          re = hb[2 * h2];
          im = -hb[2 * h2 + 1];
        }
        sk[2 * id] = re / n;
        sk[2 * id + 1] = im / n;
      }
  return TILD_OK;
}

// ---- schedule tuning -------------------------------------------------------------------------
void get_tune(const tild_ctx* c, tild_tune* t) {
  t->spread_mode = c->spread_mode;
  t->spread_cap = c->spread_cap;
  t->sort_interval = c->sort_interval;
  t->fft_streams = c->lanes;
  t->gather_mode = c->gather_mode;
  t->gather_cap = c->gather_cap;
  t->sort_brick = c->sort_brick;
  t->field_layout = c->field_layout;
  t->fft_pipeline = c->fft_pipeline;
  t->spread_ahead = c->spread_ahead;
  t->ms_per_step = 0.0;
}

int set_tune(tild_ctx* c, const tild_tune* t) {
  if (!t || (t->spread_mode != TILD_SPREAD_TILED && t->spread_mode != TILD_SPREAD_DIRECT) || t->spread_cap < 1024 ||
      t->spread_cap > 12288 || (t->spread_cap & 3) || t->sort_interval < 0 || t->fft_streams < 0 || t->fft_streams > 8 ||
      t->gather_mode < TILD_GATHER_DIRECT || t->gather_mode > TILD_GATHER_BOX || t->gather_cap < 1024 ||
      t->gather_cap > 3072 || t->field_layout < TILD_FIELD_LINEAR || t->field_layout > TILD_FIELD_BRICK ||
      (t->field_layout == TILD_FIELD_BRICK && c->D != 3) || t->fft_pipeline < 0 || t->fft_pipeline > 2 ||
      t->spread_ahead < 0 || t->spread_ahead > 1)
    return set_err(c, TILD_ERR_BAD_INPUT, "tune values out of range");
  if (t->sort_interval > 0 && !c->sort_temp) return set_err(c, TILD_ERR_UNSUPPORTED, "the context was created without sorting");
  {
    const auto cand = tild_brick_candidates(c->D);
    if (std::find(cand.begin(), cand.end(), (int)t->sort_brick) == cand.end())
      return set_err(c, TILD_ERR_BAD_INPUT, "sort_brick is not one of the supported brick shapes");
  }
  cudaSetDevice(c->device);
  if (tild_check(c, cudaStreamSynchronize(c->stream), "sync before tune")) return TILD_ERR_CUDA;
  c->spread_mode = t->spread_mode;
  c->spread_cap = t->spread_cap;
  c->gather_mode = t->gather_mode;
  c->gather_cap = t->gather_cap;
  c->field_layout = t->field_layout;
  c->fft_pipeline = t->fft_pipeline;
  c->spread_ahead = t->spread_ahead;
  if (t->sort_brick != c->sort_brick) {
    c->sort_brick = t->sort_brick;
    c->steps_since_sort = c->sort_interval;  // re-sort with the new keys at the next step
  }
  if (t->sort_interval != c->sort_interval) {
    c->sort_interval = t->sort_interval;
    c->steps_since_sort = c->sort_interval;
  }
  if (tild_assign_lanes(c, t->fft_streams)) return TILD_ERR_CUDA;
  // captured graphs hold the old launches
  for (auto& ge : c->graphs) cudaGraphExecDestroy(ge.exec);
  c->graphs.clear();
  return TILD_OK;
}

int engine_autotune(tild_ctx* c, int trial_steps, tild_tune* best) {
  if (!c || trial_steps < 1) return TILD_ERR_BAD_INPUT;
  if (c->rng == TILD_RNG_XORWOW) return set_err(c, TILD_ERR_UNSUPPORTED, "autotuning would advance the cuRAND states");
  if (!all_ready(c)) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  // snapshot every system with a state
  struct Snap {
    std::vector<float> x, xo, nz;
    int64_t step;
    bool active;
  };
  std::vector<Snap> snap(c->nsys);
  for (int s = 0; s < c->nsys; s++) {
    SysHost& h = c->sys[s];
    snap[s].step = h.step;
    snap[s].active = h.active;
    if (!h.state_set) continue;
    const size_t n = (size_t)h.ns * h.D;
    snap[s].x.resize(n);
    snap[s].xo.resize(n);
    snap[s].nz.resize(n);
    int rc = sys_get_state(c, s, snap[s].x.data(), snap[s].xo.data(), snap[s].nz.data());
    if (rc) return rc;
  }
  const bool use_graphs = c->use_graphs;
  int rc = TILD_OK;
  auto trial = [&](const tild_tune& t, double* ms) -> int {
    int r = set_tune(c, &t);
    if (r) return r;
    const int period = c->sort_interval > 0 ? 2 * c->sort_interval : c->graph_len;
    r = run_steps(c, period);  // warm-up (and graph capture)
    if (r) return r;
    return engine_time(c, trial_steps, ms);
  };
  tild_tune cur;
  get_tune(c, &cur);
  double cur_ms = 0.0;
  rc = trial(cur, &cur_ms);
  auto consider = [&](tild_tune t) {
    if (rc) return;
    double ms = 0.0;
    rc = trial(t, &ms);
    if (!rc && ms < cur_ms) {
      cur = t;
      cur_ms = ms;
    }
  };
  if (c->P >= 2) {
    for (int mode : {TILD_SPREAD_TILED, TILD_SPREAD_DIRECT}) {
      tild_tune t = cur;
      t.spread_mode = mode;
      if (mode != cur.spread_mode) consider(t);
    }
    if (cur.spread_mode == TILD_SPREAD_TILED)
      for (int cap : {3072, 6144, 12288}) {
        tild_tune t = cur;
        t.spread_cap = cap;
        if (cap != cur.spread_cap) consider(t);
      }
    if (c->D == 3)
      for (int layout : {TILD_FIELD_LINEAR, TILD_FIELD_BRICK}) {
        tild_tune t = cur;
        t.field_layout = layout;
        if (layout != cur.field_layout) consider(t);
      }
    for (int mode : {TILD_GATHER_DIRECT, TILD_GATHER_BOX}) {
      tild_tune t = cur;
      t.gather_mode = mode;
      if (mode == TILD_GATHER_BOX && cur.field_layout != TILD_FIELD_LINEAR) continue;  // box reads the linear field
      if (mode != cur.gather_mode) consider(t);
    }
    if (cur.gather_mode != TILD_GATHER_DIRECT)
      for (int cap : {1536, 2048, 3072}) {
        tild_tune t = cur;
        t.gather_cap = cap;
        if (cap != cur.gather_cap) consider(t);
      }
  }
  for (int sa : {0, 1}) {
    tild_tune t = cur;
    t.spread_ahead = sa;
    if (sa != cur.spread_ahead) consider(t);
  }
  if (c->sort_temp)
    for (int brick : tild_brick_candidates(c->D)) {
      tild_tune t = cur;
      t.sort_brick = brick;
      if (brick != cur.sort_brick) consider(t);
    }
  if (c->sort_temp)
    for (int si : {8, 16, 32}) {
      tild_tune t = cur;
      t.sort_interval = si;
      if (si != cur.sort_interval) consider(t);
    }
  if (!c->aux.empty()) {
    for (int l : {0, 2, 4, 8}) {
      tild_tune t = cur;
      t.fft_streams = std::min<int>(l, (int)c->aux.size());
      if (t.fft_streams != cur.fft_streams) consider(t);
    }
    for (int pl : {0, 1, 2}) {
      tild_tune t = cur;
      t.fft_pipeline = pl;
      if (pl != cur.fft_pipeline) consider(t);
    }
  }
  const int rc_trials = rc;
  // keep the fastest, then put every system back where it was
  rc = set_tune(c, &cur);
  for (int s = 0; s < c->nsys && !rc; s++) {
    SysHost& h = c->sys[s];
    h.active = snap[s].active;
    if (!snap[s].x.empty()) rc = sys_set_state(c, s, snap[s].x.data(), snap[s].xo.data(), snap[s].nz.data());
    if (!rc) {
      h.step = snap[s].step;
      c->h_sys[s].step = snap[s].step;
    }
  }
  if (!rc) rc = tild_upload_sys(c);
  c->use_graphs = use_graphs;
  if (rc_trials) return rc_trials;
  if (rc) return rc;
  if (best) {
    *best = cur;
    best->ms_per_step = cur_ms / trial_steps;
  }
  return TILD_OK;
}

// ---- asynchronous snapshots ------------------------------------------------------------------
int snap_setup(tild_ctx* c) {
  if (c->snap_stream) return TILD_OK;
  size_t nx = 1, nr = 1;
  for (const SysHost& h : c->sys) {
    nx = std::max(nx, (size_t)h.cap * h.D);
    nr = std::max(nr, (size_t)((h.T + h.C) * h.g.M));
  }
  if (tild_check(c, cudaStreamCreateWithFlags(&c->snap_stream, cudaStreamNonBlocking), "snapshot stream"))
    return TILD_ERR_CUDA;
  for (auto& sl : c->snaps) {
    if (tild_check(c, cudaMalloc(&sl.dx, nx * sizeof(float)), "alloc snapshot") ||
        tild_check(c, cudaMalloc(&sl.drho, nr * sizeof(float)), "alloc snapshot"))
      return TILD_ERR_OOM;
    if (tild_check(c, cudaEventCreateWithFlags(&sl.captured, cudaEventDisableTiming), "snapshot event") ||
        tild_check(c, cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "snapshot event"))
      return TILD_ERR_CUDA;
  }
  c->snap_x_floats = nx;
  c->snap_rho_floats = nr;
  return TILD_OK;
}

int sys_snapshot_async(tild_ctx* c, int s, float* x, float* rho, int64_t* ticket) {
  if (check_sys(c, s) || (!x && !rho)) return TILD_ERR_BAD_INPUT;
  SysHost& h = c->sys[s];
  if (x && !h.state_set) return set_err(c, TILD_ERR_STATE, "no state");
  if (rho && !h.have_forces) return set_err(c, TILD_ERR_STATE, "no force evaluation yet");
  cudaSetDevice(c->device);
  int rc = snap_setup(c);
  if (rc) return rc;
  const long long t = c->snap_next;
  auto& sl = c->snaps[t % TILD_SNAPSHOT_SLOTS];
  // the slot's previous copy must have left its device buffers before they are overwritten
  if (sl.ticket.load() >= 0 && tild_check(c, cudaEventSynchronize(sl.done), "snapshot slot")) return TILD_ERR_CUDA;
  const size_t n = (size_t)h.ns * h.D;
  const size_t nr = (size_t)(h.T + h.C) * h.g.M;
  if (x) {
    k_unpack_pos<<<nblk(h.ns_pad, 256), 256, 0, c->stream>>>(c->pos[c->cur] + h.slot0, c->bead_id + h.slot0,
                                                             h.ns_pad, h.D, sl.dx);
    c->launches++;
  }
  if (rho && tild_density_planar(c, s, sl.drho, c->stream)) return TILD_ERR_CUDA;
  if (tild_check(c, cudaEventRecord(sl.captured, c->stream), "snapshot event") ||
      tild_check(c, cudaStreamWaitEvent(c->snap_stream, sl.captured, 0), "snapshot wait"))
    return TILD_ERR_CUDA;
  if ((x && tild_check(c, cudaMemcpyAsync(x, sl.dx, n * sizeof(float), cudaMemcpyDeviceToHost, c->snap_stream),
                       "snapshot x")) ||
      (rho && tild_check(c, cudaMemcpyAsync(rho, sl.drho, nr * sizeof(float), cudaMemcpyDeviceToHost, c->snap_stream),
                         "snapshot rho")))
    return TILD_ERR_CUDA;
  if (tild_check(c, cudaEventRecord(sl.done, c->snap_stream), "snapshot event")) return TILD_ERR_CUDA;
  sl.ticket.store(t);
  c->snap_next = t + 1;
  if (ticket) *ticket = t;
  return TILD_OK;
}

// Safe from a writer thread: it reads only the slot's ticket (atomic) and its completion event.
int snapshot_wait(tild_ctx* c, int64_t ticket) {
  if (!c || ticket < 0) return TILD_ERR_BAD_INPUT;
  auto& sl = c->snaps[ticket % TILD_SNAPSHOT_SLOTS];
  const long long held = sl.ticket.load();
  if (held < 0 || ticket > held) return TILD_ERR_BAD_INPUT;  // never issued
  if (ticket < held) return TILD_OK;  // the slot was reused, which waited for this copy first
  cudaSetDevice(c->device);
  const cudaError_t e = cudaEventSynchronize(sl.done);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return TILD_ERR_CUDA;
  }
  return TILD_OK;
}

}  // namespace

struct tild_batch : public tild_ctx {};

// The previous step's gather spread positions that the host is about to replace (or whose types,
// charges or box change): clear the accumulator so that the next step spreads afresh.
int tild_drop_ahead(tild_ctx* c) {
  if (!c->rho_ahead) return TILD_OK;
  c->rho_ahead = false;
  return tild_check(c, cudaMemsetAsync(c->rho_fx, 0, sizeof(unsigned long long) * c->grid_total, c->stream),
                    "clear density accumulator");
}

int tild_upload_sys(tild_ctx* c) {
  for (int s = 0; s < c->nsys; s++) c->h_sys[s].active = c->sys[s].active ? 1 : 0;
  if (tild_check(c, cudaMemcpyAsync(c->d_sys, c->h_sys.data(), sizeof(SysDev) * c->nsys, cudaMemcpyHostToDevice, c->stream), "upload descriptors") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync descriptors"))
    return TILD_ERR_CUDA;
  return TILD_OK;
}

int tild_check(tild_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return 0;
  cudaGetLastError();
  if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return 1;
}

int tild_check_fft(tild_ctx* c, cufftResult r, const char* what) {
  if (r == CUFFT_SUCCESS) return 0;
  char buf[128];
  snprintf(buf, sizeof buf, "%s: cuFFT error %d", what, (int)r);
  if (c) c->err = buf;
  return 1;
}

int tild_poll_status(tild_ctx* c) {
  int st = 0;
  if (tild_check(c, cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "status") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync"))
    return TILD_ERR_CUDA;
  if (st & ST_NONFINITE_POS) return set_err(c, TILD_ERR_NAN, "non-finite bead position");
  if (st & ST_INDEX_RANGE) return set_err(c, TILD_ERR_BAD_INPUT, "bead position outside [-L, 2L): grid index out of range");
  if (st & ST_NLIST_OVERFLOW) {
    cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream);
    return set_err(c, TILD_ERR_BAD_INPUT, "neighbour list: more entries than CELL_MAX");
  }
  return TILD_OK;
}

extern "C" {

int32_t tild_abi_version(void) { return TILD_ABI_VERSION; }

const char* tild_status_string(int32_t s) {
  switch (s) {
    case TILD_OK: return "ok";
    case TILD_ERR_CUDA: return "CUDA error";
    case TILD_ERR_NAN: return "non-finite value";
    case TILD_ERR_OOM: return "out of device memory";
    case TILD_ERR_TIMEOUT: return "device wait timed out";
    case TILD_ERR_BAD_INPUT: return "bad input";
    case TILD_ERR_UNSUPPORTED: return "unsupported configuration";
    case TILD_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

const char* tild_last_error(const tild_ctx* c) { return c ? c->err.c_str() : "null context"; }

static int create_common(const tild_config* cfgs, int nsys, int device, tild_batch** out,
                         const int32_t* capacity = nullptr) {
  if (!cfgs || !out || nsys < 1) return TILD_ERR_BAD_INPUT;
  *out = nullptr;
  tild_batch* c = new tild_batch();
  const int rc = engine_create(cfgs, nsys, device, c, capacity);
  if (rc) {
    fprintf(stderr, "tild_create: %s\n", c->err.c_str());
    free_all(c);
    delete c;
    return rc;
  }
  *out = c;
  return TILD_OK;
}

int32_t tild_create(const tild_config* cfg, int32_t device, tild_ctx** out) {
  if (!cfg || !out) return TILD_ERR_BAD_INPUT;
  tild_batch* b = nullptr;
  const int rc = create_common(cfg, 1, device, &b);
  *out = b;
  return rc;
}

int32_t tild_destroy(tild_ctx* c) {
  if (!c) return TILD_ERR_BAD_INPUT;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  delete static_cast<tild_batch*>(c);
  return TILD_OK;
}

int32_t tild_set_topology(tild_ctx* c, const int32_t* types, const float* charges, const int32_t* n_bonds,
                          const int32_t* bonded_to, const int32_t* bond_type) {
  return sys_set_topology(c, 0, types, charges, n_bonds, bonded_to, bond_type);
}

int32_t tild_set_state(tild_ctx* c, const float* x, const float* xo, const float* prev_noise) {
  return sys_set_state(c, 0, x, xo, prev_noise);
}

int32_t tild_get_state(tild_ctx* c, float* x, float* xo, float* prev_noise) { return sys_get_state(c, 0, x, xo, prev_noise); }

int32_t tild_forces(tild_ctx* c, float* f) { return sys_forces(c, 0, f); }

int32_t tild_step(tild_ctx* c, int32_t nsteps) {
  if (!c || nsteps < 0) return TILD_ERR_BAD_INPUT;
  return engine_step(c, nsteps);
}

int32_t tild_get_step(tild_ctx* c, int64_t* step) {
  if (!c || !step) return TILD_ERR_BAD_INPUT;
  *step = c->sys[0].step;
  return TILD_OK;
}

int32_t tild_set_step(tild_ctx* c, int64_t step) { return sys_set_step(c, 0, step); }

int32_t tild_observables(tild_ctx* c, tild_obs* o) { return sys_observables(c, 0, o); }

int32_t tild_get_density(tild_ctx* c, float* rho) { return sys_density(c, 0, rho); }

int32_t tild_get_stencil(tild_ctx* c, int32_t* inds, float* w) {
  if (!c) return TILD_ERR_BAD_INPUT;
  const SysHost& h = c->sys[0];
  if (!h.state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  const size_t n = (size_t)h.ns * h.S;
  int* di = nullptr;
  float* dw = nullptr;
  int rc = TILD_OK;
  if (inds && dalloc(c, &di, n, "stencil indices")) rc = TILD_ERR_OOM;
  if (!rc && w && dalloc(c, &dw, n, "stencil weights")) rc = TILD_ERR_OOM;
  if (!rc) rc = tild_stencil_run(c, 0, di, dw);
  if (!rc && inds && tild_check(c, cudaMemcpyAsync(inds, di, n * 4, cudaMemcpyDeviceToHost, c->stream), "download")) rc = TILD_ERR_CUDA;
  if (!rc && w && tild_check(c, cudaMemcpyAsync(w, dw, n * 4, cudaMemcpyDeviceToHost, c->stream), "download")) rc = TILD_ERR_CUDA;
  if (!rc && tild_check(c, cudaStreamSynchronize(c->stream), "sync")) rc = TILD_ERR_CUDA;
  cudaFree(di);
  cudaFree(dw);
  return rc ? rc : tild_poll_status(c);
}

int32_t tild_sk_accumulate(tild_ctx* c, int32_t slot, int32_t type) { return sys_sk_accumulate(c, 0, slot, type); }

int32_t tild_sk_get(tild_ctx* c, int32_t slot, double* sk, int32_t* ncalls) { return sys_sk_get(c, 0, slot, sk, ncalls); }

int32_t tild_nlist_build(tild_ctx* c, float rc, int32_t group_type, int32_t* cell_of, int32_t* neigh_count,
                         int32_t* neigh, int32_t* cell_max_out) {
  if (!c || !(rc > 0.f) || group_type < -1 || group_type >= c->sys[0].T) return TILD_ERR_BAD_INPUT;
  const SysHost& h = c->sys[0];
  if (!h.state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  int nc[3], total, cmax;
  float Lc[3];
  if (tild_nlist_geom(h, rc, nc, Lc, &total, &cmax)) return set_err(c, TILD_ERR_BAD_INPUT, "cutoff larger than the box");
  if (cell_max_out) *cell_max_out = cmax;
  if (!cell_of && !neigh_count && !neigh) return TILD_OK;
  const size_t ns = h.ns;
  int *dc = nullptr, *dn = nullptr, *dl = nullptr;
  int r = TILD_OK;
  if (dalloc(c, &dc, ns, "nlist") || dalloc(c, &dn, ns, "nlist") || dalloc(c, &dl, ns * (size_t)std::max(cmax, 1), "nlist"))
    r = TILD_ERR_OOM;
  if (!r) r = tild_nlist_run(c, 0, rc, group_type, dc, dn, dl);
  int st = r ? r : tild_poll_status(c);
  if (!r) {
    if ((cell_of && tild_check(c, cudaMemcpy(cell_of, dc, ns * 4, cudaMemcpyDeviceToHost), "download")) ||
        (neigh_count && tild_check(c, cudaMemcpy(neigh_count, dn, ns * 4, cudaMemcpyDeviceToHost), "download")) ||
        (neigh && tild_check(c, cudaMemcpy(neigh, dl, ns * (size_t)cmax * 4, cudaMemcpyDeviceToHost), "download")))
      r = TILD_ERR_CUDA;
  }
  cudaFree(dc);
  cudaFree(dn);
  cudaFree(dl);
  return r ? r : st;
}

int32_t tild_time_steps(tild_ctx* c, int32_t nsteps, double* ms) { return engine_time(c, nsteps, ms); }

int32_t tild_profile_steps(tild_ctx* c, int32_t nsteps, double* stage_ms, int32_t max_stages, int32_t* n_stages,
                           char* names, int32_t name_cap) {
  if (!c || !stage_ms || nsteps < 0) return TILD_ERR_BAD_INPUT;
  if (!all_ready(c)) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  c->prof_ev.clear();
  c->prof_stage.clear();
  c->profiling = true;
  int rc = TILD_OK;
  for (int k = 0; k < nsteps && !rc; k++) rc = tild_run_forces(c, true, nullptr, -1);
  c->profiling = false;
  cudaEvent_t last;
  cudaEventCreate(&last);
  cudaEventRecord(last, c->stream);
  cudaEventSynchronize(last);
  double acc[STAGE_COUNT] = {0};
  for (size_t i = 0; i < c->prof_ev.size(); i++) {
    const cudaEvent_t end = (i + 1 < c->prof_ev.size()) ? c->prof_ev[i + 1] : last;
    float t = 0.f;
    cudaEventElapsedTime(&t, c->prof_ev[i], end);
    acc[c->prof_stage[i]] += t;
  }
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  cudaEventDestroy(last);
  c->prof_ev.clear();
  c->prof_stage.clear();
  const int n = std::min<int>(max_stages, STAGE_COUNT);
  for (int i = 0; i < n; i++) stage_ms[i] = acc[i];
  if (n_stages) *n_stages = n;
  if (names && name_cap > 0) {
    std::string s;
    for (int i = 0; i < n; i++) {
      if (i) s += ",";
      s += kStageNames[i];
    }
    snprintf(names, (size_t)name_cap, "%s", s.c_str());
  }
  return rc ? rc : tild_poll_status(c);
}

int32_t tild_kernel_launches(tild_ctx* c, int64_t* count) {
  if (!c || !count) return TILD_ERR_BAD_INPUT;
  *count = c->launches;
  return TILD_OK;
}

int32_t tild_sync(tild_ctx* c) {
  if (!c) return TILD_ERR_BAD_INPUT;
  cudaSetDevice(c->device);
  return tild_poll_status(c);
}

// ---- batches ------------------------------------------------------------------------------
int32_t tild_batch_create(const tild_config* cfgs, int32_t nsys, int32_t device, tild_batch** out) {
  return create_common(cfgs, nsys, device, out);
}
int32_t tild_batch_create_slots(const tild_config* cfgs, const int32_t* capacity, int32_t nsys, int32_t device,
                                tild_batch** out) {
  if (!capacity) return TILD_ERR_BAD_INPUT;
  return create_common(cfgs, nsys, device, out, capacity);
}
int32_t tild_batch_load(tild_batch* b, int32_t sys, const tild_config* cfg) { return sys_load(b, sys, cfg); }
int32_t tild_autotune(tild_ctx* c, int32_t trial_steps, tild_tune* best) { return engine_autotune(c, trial_steps, best); }
int32_t tild_snapshot_async(tild_ctx* c, float* x, float* rho, int64_t* ticket) {
  if (!c) return TILD_ERR_BAD_INPUT;
  return sys_snapshot_async(c, 0, x, rho, ticket);
}
int32_t tild_snapshot_wait(tild_ctx* c, int64_t ticket) { return snapshot_wait(c, ticket); }
int32_t tild_batch_snapshot_async(tild_batch* b, int32_t sys, float* x, float* rho, int64_t* ticket) {
  if (!b) return TILD_ERR_BAD_INPUT;
  return sys_snapshot_async(b, sys, x, rho, ticket);
}
int32_t tild_batch_snapshot_wait(tild_batch* b, int64_t ticket) { return snapshot_wait(b, ticket); }
void* tild_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void tild_host_free(void* p) {
  if (p) cudaFreeHost(p);
}
int32_t tild_get_tune(tild_ctx* c, tild_tune* out) {
  if (!c || !out) return TILD_ERR_BAD_INPUT;
  get_tune(c, out);
  return TILD_OK;
}
int32_t tild_set_tune(tild_ctx* c, const tild_tune* t) {
  if (!c) return TILD_ERR_BAD_INPUT;
  return set_tune(c, t);
}
int32_t tild_batch_autotune(tild_batch* b, int32_t trial_steps, tild_tune* best) { return engine_autotune(b, trial_steps, best); }
int32_t tild_batch_get_tune(tild_batch* b, tild_tune* out) { return tild_get_tune(b, out); }
int32_t tild_batch_set_tune(tild_batch* b, const tild_tune* t) { return tild_set_tune(b, t); }
int32_t tild_batch_capacity(tild_batch* b, int32_t sys, int32_t* capacity) {
  if (check_sys(b, sys) || !capacity) return TILD_ERR_BAD_INPUT;
  *capacity = b->sys[sys].cap;
  return TILD_OK;
}
int32_t tild_batch_set_stop(tild_batch* b, int32_t sys, int64_t stop_at) {
  if (check_sys(b, sys) || stop_at < -1) return TILD_ERR_BAD_INPUT;
  b->h_sys[sys].stop_at = stop_at;
  if (stop_at >= 0) b->any_stop = true;
  return tild_upload_sys(b);
}
int32_t tild_batch_get_active(tild_batch* b, int32_t sys, int32_t* active) {
  if (check_sys(b, sys) || !active) return TILD_ERR_BAD_INPUT;
  *active = b->sys[sys].active ? 1 : 0;
  return TILD_OK;
}
int32_t tild_batch_sk_accumulate(tild_batch* b, int32_t sys, int32_t slot, int32_t type) {
  return sys_sk_accumulate(b, sys, slot, type);
}
int32_t tild_batch_sk_get(tild_batch* b, int32_t sys, int32_t slot, double* sk, int32_t* ncalls) {
  return sys_sk_get(b, sys, slot, sk, ncalls);
}
int32_t tild_batch_destroy(tild_batch* b) { return tild_destroy(b); }
const char* tild_batch_last_error(const tild_batch* b) { return tild_last_error(b); }
int32_t tild_batch_set_topology(tild_batch* b, int32_t sys, const int32_t* types, const float* charges,
                                const int32_t* n_bonds, const int32_t* bonded_to, const int32_t* bond_type) {
  return sys_set_topology(b, sys, types, charges, n_bonds, bonded_to, bond_type);
}
int32_t tild_batch_set_state(tild_batch* b, int32_t sys, const float* x, const float* xo, const float* prev_noise) {
  return sys_set_state(b, sys, x, xo, prev_noise);
}
int32_t tild_batch_get_state(tild_batch* b, int32_t sys, float* x, float* xo, float* prev_noise) {
  return sys_get_state(b, sys, x, xo, prev_noise);
}
int32_t tild_batch_set_active(tild_batch* b, int32_t sys, int32_t active) {
  if (check_sys(b, sys)) return TILD_ERR_BAD_INPUT;
  if (active && b->h_sys[sys].stop_at >= 0 && b->sys[sys].step >= b->h_sys[sys].stop_at)
    return set_err(b, TILD_ERR_STATE, "the system is at or past its stop step");
  b->sys[sys].active = active != 0;
  return tild_upload_sys(b);
}
int32_t tild_batch_set_step(tild_batch* b, int32_t sys, int64_t step) { return sys_set_step(b, sys, step); }
int32_t tild_batch_get_step(tild_batch* b, int32_t sys, int64_t* step) {
  if (check_sys(b, sys) || !step) return TILD_ERR_BAD_INPUT;
  *step = b->sys[sys].step;
  return TILD_OK;
}
int32_t tild_batch_step(tild_batch* b, int32_t nsteps) {
  if (!b || nsteps < 0) return TILD_ERR_BAD_INPUT;
  return engine_step(b, nsteps);
}
int32_t tild_batch_forces(tild_batch* b, int32_t sys, float* f) { return sys_forces(b, sys, f); }
int32_t tild_batch_observables(tild_batch* b, int32_t sys, tild_obs* o) { return sys_observables(b, sys, o); }
int32_t tild_batch_get_density(tild_batch* b, int32_t sys, float* rho) { return sys_density(b, sys, rho); }
int32_t tild_batch_time_steps(tild_batch* b, int32_t nsteps, double* ms) { return engine_time(b, nsteps, ms); }
int32_t tild_batch_sync(tild_batch* b) { return tild_sync(b); }

}  // extern "C"
