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

// pack positions [ns][D] (bead order) into float4 slots with the type in .w
__global__ void k_pack_pos(const float* __restrict__ x, const int* __restrict__ types, const int* __restrict__ slot_of,
                           int ns, int D, float4* __restrict__ pos) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= ns) return;
  const float* xb = x + (long long)b * D;
  pos[slot_of[b]] = make_float4(xb[0], xb[1], D == 3 ? xb[2] : 0.f, __int_as_float(types[b] & 0xff));
}

__global__ void k_pack_noise(const float* __restrict__ src, const int* __restrict__ slot_of, int ns, int D,
                             float* __restrict__ noise) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= ns) return;
  const int s = slot_of[b];
  for (int d = 0; d < 3; d++) noise[3 * (long long)s + d] = (src && d < D) ? src[(long long)b * D + d] : 0.f;
}

__global__ void k_unpack_pos(const float4* __restrict__ pos, const int* __restrict__ bead_id, int ns, int D,
                             float* __restrict__ x) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const float4 p = pos[s];
  float* xb = x + (long long)bead_id[s] * D;
  xb[0] = p.x;
  xb[1] = p.y;
  if (D == 3) xb[2] = p.z;
}

__global__ void k_unpack_noise(const float* __restrict__ noise, const int* __restrict__ bead_id, int ns, int D,
                               float* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  for (int d = 0; d < D; d++) out[(long long)bead_id[s] * D + d] = noise[3 * (long long)s + d];
}

__global__ void k_init_xorwow(curandStateXORWOW_t* st, const int* __restrict__ bead_id, int ns, unsigned int seed) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
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
                  c->bondk_dev, c->bondr_dev, c->types_dev, c->xorwow, c->rho, c->rhok, c->gk, c->gfield, c->utab,
                  c->ctab, c->virk, c->frfield, c->rho_fx, c->g4, c->kd, c->kk, c->red, c->xfer, c->d_status};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int i = 0; i < TILD_MAX_COMPUTES; i++)
    if (c->sk[i]) cudaFree(c->sk[i]);
  if (c->plans) {
    cufftDestroy(c->plan_r2c);
    cufftDestroy(c->plan_c2r);
  }
  tild_sort_free(c);
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

}  // namespace

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

int32_t tild_create(const tild_config* cfg, int32_t device, tild_ctx** out) {
  if (!cfg || !out) return TILD_ERR_BAD_INPUT;
  *out = nullptr;
  std::string why;
  int v = validate(cfg, why);
  if (v) {
    fprintf(stderr, "tild_create: %s\n", why.c_str());
    return v;
  }
  tild_ctx* c = new tild_ctx();
  c->cfg = *cfg;
  c->device = device;
  if (tild_check(c, cudaSetDevice(device), "cudaSetDevice")) {
    fprintf(stderr, "tild_create: %s\n", c->err.c_str());
    delete c;
    return TILD_ERR_CUDA;
  }
  if (tild_check(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) {
    delete c;
    return TILD_ERR_CUDA;
  }
  c->D = cfg->dim;
  c->T = cfg->ntypes;
  c->C = cfg->do_charges ? 1 : 0;
  c->ns = cfg->ns;
  c->p = cfg->pmeorder;
  c->nP = (c->D == 2) ? 3 : 6;
  c->max_steps = cfg->max_steps;
  Geom& g = c->g;
  g.M = 1;
  c->S = 1;
  float gv = 1.0f;
  for (int d = 0; d < 3; d++) {
    g.nx[d] = (d < c->D) ? cfg->nx[d] : 1;
    g.L[d] = (d < c->D) ? cfg->box[d] : 1.0f;
    g.Lh[d] = 0.5f * g.L[d];
    g.dx[d] = g.L[d] / (float)g.nx[d];
  }
  c->dV = 1.0;
  c->V = 1.0;
  for (int d = 0; d < c->D; d++) {
    gv *= g.dx[d];
    g.M *= g.nx[d];
    c->S *= (c->p + 1);
    c->dV *= (double)g.dx[d];
    c->V *= (double)g.L[d];
  }
  g.gvol = gv;
  g.nxh = g.nx[0] / 2 + 1;
  g.Mh = g.M / g.nx[0] * g.nxh;

  // style bookkeeping: FFT styles get a table slot, fieldphases a static field
  c->fft_style_index.assign(cfg->n_styles, -1);
  for (int i = 0; i < cfg->n_styles; i++) {
    const tild_pair_style& s = cfg->styles[i];
    if (s.style == TILD_STYLE_FIELDPHASE) {
      FieldK f;
      f.a = s.type1;
      f.b = s.type2;
      f.slot = i;
      c->fields.push_back(f);
    } else {
      StyleK k;
      k.a = s.type1;
      k.b = s.type2;
      k.ramp = s.ramp;
      k.Ai = s.prefactor;
      k.Af = s.final_prefactor;
      k.uk0 = 1.0f;
      c->fft_style_index[i] = (int)c->styles_k.size();
      c->fft_style_cfg.push_back(i);
      c->styles_k.push_back(k);
    }
  }
  for (int t = 0; t < c->T; t++) {
    int m = 0;
    for (int k = 0; k < cfg->n_integrators; k++)
      if (cfg->integrators[k].group_type < 0 || cfg->integrators[k].group_type == t) m |= 1 << k;
    c->type_integ_mask[t] = m;
  }

  const size_t ns = c->ns, M = g.M, Mh = g.Mh;
  c->spread_cap = 12288;
  const size_t nch = c->T + c->C;
  const size_t nfft = c->styles_k.size();
  int rc = TILD_OK;
  rc = rc ? rc : dalloc(c, &c->pos[0], ns, "positions");
  rc = rc ? rc : dalloc(c, &c->pos[1], ns, "positions");
  rc = rc ? rc : dalloc(c, &c->noise, ns * 3, "noise");
  rc = rc ? rc : dalloc(c, &c->bead_id, ns, "bead ids");
  rc = rc ? rc : dalloc(c, &c->slot_of, ns, "slots");
  rc = rc ? rc : dalloc(c, &c->bond_nbr, ns * 3, "bonds");
  rc = rc ? rc : dalloc(c, &c->bond_info, ns, "bonds");
  rc = rc ? rc : dalloc(c, &c->types_dev, ns, "types");
  rc = rc ? rc : dalloc(c, &c->bondk_dev, TILD_MAX_BOND_TYPES, "bond constants");
  rc = rc ? rc : dalloc(c, &c->bondr_dev, TILD_MAX_BOND_TYPES, "bond constants");
  if (c->C) rc = rc ? rc : dalloc(c, &c->charge, ns, "charges");
  rc = rc ? rc : dalloc(c, &c->rho, nch * M, "densities");
  rc = rc ? rc : dalloc(c, &c->rho_fx, nch * M, "density accumulator");
  rc = rc ? rc : dalloc(c, &c->rhok, nch * Mh, "density spectra");
  rc = rc ? rc : dalloc(c, &c->gk, nch * c->D * Mh, "force spectra");
  rc = rc ? rc : dalloc(c, &c->gfield, nch * c->D * M, "force fields");
  rc = rc ? rc : dalloc(c, &c->g4, nch * M, "interleaved force fields");
  rc = rc ? rc : dalloc(c, &c->utab, nfft * Mh, "multiplier tables");
  rc = rc ? rc : dalloc(c, &c->virk, nfft * c->nP * Mh, "virial tables");
  if (c->C) rc = rc ? rc : dalloc(c, &c->ctab, Mh, "charge table");
  if (!c->fields.empty()) rc = rc ? rc : dalloc(c, &c->frfield, c->fields.size() * c->D * M, "fieldphase fields");
  rc = rc ? rc : dalloc(c, &c->kd, (size_t)g.nx[0] + g.nx[1] + g.nx[2], "k vectors");
  rc = rc ? rc : dalloc(c, &c->kk, (size_t)g.nx[0] + g.nx[1] + g.nx[2], "k vectors");
  rc = rc ? rc : dalloc(c, &c->xfer, ns * 3, "transfer buffer");
  rc = rc ? rc : dalloc(c, &c->d_status, 1, "status");
  if (cfg->rng == TILD_RNG_XORWOW) rc = rc ? rc : dalloc(c, &c->xorwow, ns, "xorwow states");
  if (rc) {
    fprintf(stderr, "tild_create: %s\n", c->err.c_str());
    free_all(c);
    delete c;
    return rc;
  }
  cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream);
  cudaMemsetAsync(c->rho_fx, 0, sizeof(unsigned long long) * nch * M, c->stream);
  cudaMemsetAsync(c->noise, 0, sizeof(float) * ns * 3, c->stream);
  {
    std::vector<float> bk(TILD_MAX_BOND_TYPES, 0.f), br(TILD_MAX_BOND_TYPES, 0.f);
    for (int b = 0; b < cfg->n_bond_types; b++) {
      bk[b] = cfg->bond_k[b];
      br[b] = cfg->bond_req[b];
    }
    cudaMemcpyAsync(c->bondk_dev, bk.data(), bk.size() * 4, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->bondr_dev, br.data(), br.size() * 4, cudaMemcpyHostToDevice, c->stream);
    // identity slot order until the first sort
    std::vector<int> id(ns);
    for (size_t i = 0; i < ns; i++) id[i] = (int)i;
    cudaMemcpyAsync(c->bead_id, id.data(), ns * 4, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->slot_of, id.data(), ns * 4, cudaMemcpyHostToDevice, c->stream);
    if (tild_check(c, cudaStreamSynchronize(c->stream), "upload constants")) rc = TILD_ERR_CUDA;
  }
  // cuFFT plans: batched R2C over all density channels, batched C2R over channel x direction
  if (!rc) {
    int n[3];
    if (c->D == 3) { n[0] = g.nx[2]; n[1] = g.nx[1]; n[2] = g.nx[0]; }
    else { n[0] = g.nx[1]; n[1] = g.nx[0]; }
    if (tild_check_fft(c, cufftPlanMany(&c->plan_r2c, c->D, n, nullptr, 1, (int)M, nullptr, 1, (int)Mh, CUFFT_R2C, (int)nch), "plan R2C") ||
        tild_check_fft(c, cufftPlanMany(&c->plan_c2r, c->D, n, nullptr, 1, (int)Mh, nullptr, 1, (int)M, CUFFT_C2R, (int)(nch * c->D)), "plan C2R") ||
        tild_check_fft(c, cufftSetStream(c->plan_r2c, c->stream), "plan stream") ||
        tild_check_fft(c, cufftSetStream(c->plan_c2r, c->stream), "plan stream"))
      rc = TILD_ERR_CUDA;
    else
      c->plans = true;
  }
  c->sort_interval = cfg->sort_interval == 0 ? 16 : (cfg->sort_interval < 0 ? 0 : cfg->sort_interval);
  if (!rc && c->sort_interval > 0) rc = tild_sort_alloc(c);
  if (!rc) rc = tild_build_tables(c);
  if (rc) {
    fprintf(stderr, "tild_create: %s\n", c->err.c_str());
    free_all(c);
    delete c;
    return rc;
  }
  *out = c;
  return TILD_OK;
}

int32_t tild_destroy(tild_ctx* c) {
  if (!c) return TILD_ERR_BAD_INPUT;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  delete c;
  return TILD_OK;
}

int32_t tild_set_topology(tild_ctx* c, const int32_t* types, const float* charges, const int32_t* n_bonds,
                          const int32_t* bonded_to, const int32_t* bond_type) {
  if (!c || !types) return TILD_ERR_BAD_INPUT;
  if (c->C && !charges) return set_err(c, TILD_ERR_BAD_INPUT, "charges required when do_charges is set");
  cudaSetDevice(c->device);
  const int ns = c->ns;
  std::vector<int> slot_of(ns), bead_id(ns);
  if (tild_check(c, cudaMemcpyAsync(slot_of.data(), c->slot_of, ns * 4, cudaMemcpyDeviceToHost, c->stream), "slots") ||
      tild_check(c, cudaMemcpyAsync(bead_id.data(), c->bead_id, ns * 4, cudaMemcpyDeviceToHost, c->stream), "ids") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync"))
    return TILD_ERR_CUDA;
  std::vector<int> nbr(3 * (size_t)ns, 0), info(ns, 0);
  std::vector<float> q;
  if (c->C) q.resize(ns);
  for (int b = 0; b < ns; b++) {
    if (types[b] < 0 || types[b] >= c->T) return set_err(c, TILD_ERR_BAD_INPUT, "bead type out of range");
    const int s = slot_of[b];
    int nb = n_bonds ? n_bonds[b] : 0;
    if (nb < 0 || nb > TILD_MAX_BONDS) return set_err(c, TILD_ERR_BAD_INPUT, "more than MAX_BONDS (3) bonds on a bead");
    int in = nb;
    for (int k = 0; k < nb; k++) {
      const int j = bonded_to[3 * (size_t)b + k], bt = bond_type[3 * (size_t)b + k];
      if (j < 0 || j >= ns) return set_err(c, TILD_ERR_BAD_INPUT, "bond partner out of range");
      if (bt < 0 || bt >= c->cfg.n_bond_types) return set_err(c, TILD_ERR_BAD_INPUT, "bond type out of range");
      nbr[3 * (size_t)s + k] = slot_of[j];
      in |= bt << (8 + 8 * k);
    }
    info[s] = in;
    if (c->C) q[s] = charges[b];
  }
  if (tild_check(c, cudaMemcpyAsync(c->bond_nbr, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, c->stream), "bonds") ||
      tild_check(c, cudaMemcpyAsync(c->bond_info, info.data(), info.size() * 4, cudaMemcpyHostToDevice, c->stream), "bonds") ||
      tild_check(c, cudaMemcpyAsync(c->types_dev, types, (size_t)ns * 4, cudaMemcpyHostToDevice, c->stream), "types") ||
      (c->C && tild_check(c, cudaMemcpyAsync(c->charge, q.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, c->stream), "charges")) ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync topology"))
    return TILD_ERR_CUDA;
  // fixed-point scale of the shared-memory spread: 256 beads x the largest product of stencil
  // weights (times the largest |q| on the charge channel) must stay below 2^31
  {
    double wmax = 0.0;
    for (int k = 0; k <= 1000; k++) {
      const double sx = -0.5 + k / 1000.0;
      double W[5];
      const int P = c->p;
      double sx2 = sx * sx, sx3, sx4;
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
    double qmax = 1.0;
    if (c->C)
      for (int b = 0; b < ns; b++) qmax = std::max(qmax, (double)std::fabs(charges[b]));
    const double bound = 256.0 * std::pow(wmax * 1.05, c->D) / (double)c->g.gvol * qmax;
    int k = 0;
    while (k < 31 && bound * std::ldexp(1.0, k + 1) < 2147483647.0) k++;
    c->spread_kbits = k;
  }
  c->topo_set = true;
  return TILD_OK;
}

int32_t tild_set_state(tild_ctx* c, const float* x, const float* xo, const float* prev_noise) {
  if (!c || !x) return TILD_ERR_BAD_INPUT;
  if (!c->topo_set) return set_err(c, TILD_ERR_STATE, "tild_set_topology must come before tild_set_state");
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->ns * c->D;
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(x[i])) return set_err(c, TILD_ERR_NAN, "non-finite position in tild_set_state");
  const unsigned nb = nblk(c->ns, 256);
  if (tild_check(c, cudaMemcpyAsync(c->xfer, x, n * 4, cudaMemcpyHostToDevice, c->stream), "upload x")) return TILD_ERR_CUDA;
  k_pack_pos<<<nb, 256, 0, c->stream>>>(c->xfer, c->types_dev, c->slot_of, c->ns, c->D, c->pos[c->cur]);
  c->launches++;
  // x_{n-1}: xo when given, else x (send_3n_to_device copies x into xo, device_comm_utils.cu:15-16)
  if (xo && tild_check(c, cudaMemcpyAsync(c->xfer, xo, n * 4, cudaMemcpyHostToDevice, c->stream), "upload xo"))
    return TILD_ERR_CUDA;
  k_pack_pos<<<nb, 256, 0, c->stream>>>(c->xfer, c->types_dev, c->slot_of, c->ns, c->D, c->pos[c->cur ^ 1]);
  c->launches++;
  if (prev_noise && tild_check(c, cudaMemcpyAsync(c->xfer, prev_noise, n * 4, cudaMemcpyHostToDevice, c->stream), "upload noise"))
    return TILD_ERR_CUDA;
  k_pack_noise<<<nb, 256, 0, c->stream>>>(prev_noise ? c->xfer : nullptr, c->slot_of, c->ns, c->D, c->noise);
  c->launches++;
  if (c->cfg.rng == TILD_RNG_XORWOW) {
    k_init_xorwow<<<nb, 256, 0, c->stream>>>(c->xorwow, c->bead_id, c->ns, (unsigned int)c->cfg.seed);
    c->launches++;
  }
  if (c->sort_interval > 0) {
    int rs = tild_sort_beads(c);
    if (rs) return rs;
  }
  if (tild_check(c, cudaStreamSynchronize(c->stream), "set state")) return TILD_ERR_CUDA;
  c->state_set = true;
  c->have_forces = false;
  return TILD_OK;
}

int32_t tild_get_state(tild_ctx* c, float* x, float* xo, float* prev_noise) {
  if (!c) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->ns * c->D;
  const unsigned nb = nblk(c->ns, 256);
  float* outs[3] = {x, xo, prev_noise};
  for (int k = 0; k < 3; k++) {
    if (!outs[k]) continue;
    if (k < 2) k_unpack_pos<<<nb, 256, 0, c->stream>>>(c->pos[k == 0 ? c->cur : c->cur ^ 1], c->bead_id, c->ns, c->D, c->xfer);
    else k_unpack_noise<<<nb, 256, 0, c->stream>>>(c->noise, c->bead_id, c->ns, c->D, c->xfer);
    c->launches++;
    if (tild_check(c, cudaMemcpyAsync(outs[k], c->xfer, n * 4, cudaMemcpyDeviceToHost, c->stream), "download") ||
        tild_check(c, cudaStreamSynchronize(c->stream), "sync download"))
      return TILD_ERR_CUDA;
  }
  return TILD_OK;
}

int32_t tild_forces(tild_ctx* c, float* f) {
  if (!c) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "tild_set_state must come before tild_forces");
  cudaSetDevice(c->device);
  int rc = tild_run_forces(c, c->step, false, f ? c->xfer : nullptr);
  if (rc) return rc;
  rc = tild_poll_status(c);
  if (rc) return rc;
  if (f) {
    if (tild_check(c, cudaMemcpyAsync(f, c->xfer, (size_t)c->ns * c->D * 4, cudaMemcpyDeviceToHost, c->stream), "download f") ||
        tild_check(c, cudaStreamSynchronize(c->stream), "sync f"))
      return TILD_ERR_CUDA;
  }
  return TILD_OK;
}

int32_t tild_step(tild_ctx* c, int32_t nsteps) {
  if (!c || nsteps < 0) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "tild_set_state must come before tild_step");
  cudaSetDevice(c->device);
  for (int k = 0; k < nsteps; k++) {
    const int64_t s = c->step + 1;
    int rc = tild_run_forces(c, s, true, nullptr);
    if (rc) return rc;
    c->step = s;
  }
  return tild_poll_status(c);
}

int32_t tild_get_step(tild_ctx* c, int64_t* step) {
  if (!c || !step) return TILD_ERR_BAD_INPUT;
  *step = c->step;
  return TILD_OK;
}

int32_t tild_set_step(tild_ctx* c, int64_t step) {
  if (!c || step < 0) return TILD_ERR_BAD_INPUT;
  c->step = step;
  return TILD_OK;
}

int32_t tild_observables(tild_ctx* c, tild_obs* o) {
  if (!c || !o) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  if (!c->have_forces) {
    int rc = tild_run_forces(c, c->step, false, nullptr);
    if (rc) return rc;
  }
  int rc = tild_obs_compute(c, o);
  if (rc) return rc;
  if (!std::isfinite(o->upe)) return set_err(c, TILD_ERR_NAN, "non-finite energy");
  return tild_poll_status(c);
}

int32_t tild_get_density(tild_ctx* c, float* rho) {
  if (!c || !rho) return TILD_ERR_BAD_INPUT;
  if (!c->have_forces) return set_err(c, TILD_ERR_STATE, "no force evaluation yet");
  cudaSetDevice(c->device);
  if (tild_check(c, cudaMemcpyAsync(rho, c->rho, sizeof(float) * (size_t)(c->T + c->C) * c->g.M, cudaMemcpyDeviceToHost, c->stream), "download rho") ||
      tild_check(c, cudaStreamSynchronize(c->stream), "sync rho"))
    return TILD_ERR_CUDA;
  return TILD_OK;
}

int32_t tild_get_stencil(tild_ctx* c, int32_t* inds, float* w) {
  if (!c) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->ns * c->S;
  int* di = nullptr;
  float* dw = nullptr;
  int rc = TILD_OK;
  if (inds && dalloc(c, &di, n, "stencil indices")) rc = TILD_ERR_OOM;
  if (!rc && w && dalloc(c, &dw, n, "stencil weights")) rc = TILD_ERR_OOM;
  if (!rc) rc = tild_stencil_run(c, di, dw);
  if (!rc && inds && tild_check(c, cudaMemcpyAsync(inds, di, n * 4, cudaMemcpyDeviceToHost, c->stream), "download")) rc = TILD_ERR_CUDA;
  if (!rc && w && tild_check(c, cudaMemcpyAsync(w, dw, n * 4, cudaMemcpyDeviceToHost, c->stream), "download")) rc = TILD_ERR_CUDA;
  if (!rc && tild_check(c, cudaStreamSynchronize(c->stream), "sync")) rc = TILD_ERR_CUDA;
  cudaFree(di);
  cudaFree(dw);
  return rc ? rc : tild_poll_status(c);
}

int32_t tild_sk_accumulate(tild_ctx* c, int32_t slot, int32_t type) {
  if (!c || slot < 0 || slot >= TILD_MAX_COMPUTES || type < 0 || type >= c->T) return TILD_ERR_BAD_INPUT;
  if (!c->have_forces) return set_err(c, TILD_ERR_STATE, "no force evaluation yet");
  cudaSetDevice(c->device);
  return tild_sk_acc_run(c, slot, type);
}

int32_t tild_sk_get(tild_ctx* c, int32_t slot, double* sk, int32_t* ncalls) {
  if (!c || slot < 0 || slot >= TILD_MAX_COMPUTES) return TILD_ERR_BAD_INPUT;
  cudaSetDevice(c->device);
  const int n = c->sk[slot] ? c->sk_calls[slot] : 0;
  if (ncalls) *ncalls = n;
  if (!sk) return TILD_OK;
  const Geom& g = c->g;
  if (n == 0) {
    memset(sk, 0, sizeof(double) * 2 * (size_t)g.M);
    return TILD_OK;
  }
  std::vector<double> h(2 * (size_t)g.Mh);
  if (tild_check(c, cudaMemcpyAsync(h.data(), c->sk[slot], sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream), "download sk") ||
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
          re = h[2 * h2];
          im = h[2 * h2 + 1];
        } else {
          const int xm = N0 - x, ym = (N1 - y) % N1, zm = (N2 - z) % N2;
          const size_t h2 = (size_t)xm + (size_t)g.nxh * (ym + (size_t)N1 * zm);
          re = h[2 * h2];
          im = -h[2 * h2 + 1];
        }
        sk[2 * id] = re / n;
        sk[2 * id + 1] = im / n;
      }
  return TILD_OK;
}

int32_t tild_nlist_build(tild_ctx* c, float rc, int32_t group_type, int32_t* cell_of, int32_t* neigh_count,
                         int32_t* neigh, int32_t* cell_max_out) {
  if (!c || !(rc > 0.f) || group_type < -1 || group_type >= c->T) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  int nc[3], total, cmax;
  float Lc[3];
  if (tild_nlist_geom(c, rc, nc, Lc, &total, &cmax)) return set_err(c, TILD_ERR_BAD_INPUT, "cutoff larger than the box");
  if (cell_max_out) *cell_max_out = cmax;
  if (!cell_of && !neigh_count && !neigh) return TILD_OK;
  const size_t ns = c->ns;
  int *dc = nullptr, *dn = nullptr, *dl = nullptr;
  int r = TILD_OK;
  if (dalloc(c, &dc, ns, "nlist") || dalloc(c, &dn, ns, "nlist") || dalloc(c, &dl, ns * (size_t)std::max(cmax, 1), "nlist"))
    r = TILD_ERR_OOM;
  if (!r) r = tild_nlist_run(c, rc, group_type, dc, dn, dl);
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

int32_t tild_time_steps(tild_ctx* c, int32_t nsteps, double* ms) {
  if (!c || !ms || nsteps < 0) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  int rc = TILD_OK;
  for (int k = 0; k < nsteps && !rc; k++) {
    const int64_t s = c->step + 1;
    rc = tild_run_forces(c, s, true, nullptr);
    if (!rc) c->step = s;
  }
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc ? rc : tild_poll_status(c);
}

int32_t tild_profile_steps(tild_ctx* c, int32_t nsteps, double* stage_ms, int32_t max_stages, int32_t* n_stages,
                           char* names, int32_t name_cap) {
  if (!c || !stage_ms || nsteps < 0) return TILD_ERR_BAD_INPUT;
  if (!c->state_set) return set_err(c, TILD_ERR_STATE, "no state");
  cudaSetDevice(c->device);
  c->prof_ev.clear();
  c->prof_stage.clear();
  c->profiling = true;
  int rc = TILD_OK;
  for (int k = 0; k < nsteps && !rc; k++) {
    const int64_t s = c->step + 1;
    rc = tild_run_forces(c, s, true, nullptr);
    if (!rc) c->step = s;
  }
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

}  // extern "C"
