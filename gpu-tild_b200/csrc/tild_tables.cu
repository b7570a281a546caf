// tild_tables.cu — k-space multiplier tables, virial kernels and static fields, built once per
// context on the device.
//
// The reference builds every table in FP32 on the device (init_device_gaussian,
// pair_style_gaussian.cu:72-90; init_device_erf_kspace, pair_style_erf.cu:122-158;
// init_device_gaussian_erf, pair_style_gaussian_erf.cu:82-115; init_device_fieldphase,
// pair_style_fieldphases.cu:101-185; virial: d_initVirial + InitializeVirial,
// device_array_utils.cu:456-494 and pair_style.cu:262-276).  Here the default is FP64
// evaluation stored as FP32; TILD_TABLES_REF_FP32 evaluates the multipliers with the
// reference's FP32 expressions instead.  Tables cover only the R2C half spectrum.
#include "tild_internal.cuh"
#include <cmath>

namespace {

constexpr double kPi = 3.14159265358979323846;

// Reference FP32 constants (globals.h:29-31).
constexpr float kRefPI = 3.141592654f;
constexpr float kRefPI2 = 6.2831853071f;
constexpr float kRefPI4 = 12.56637061435917295384f;

__device__ __forceinline__ void half_index(long long h, const Geom& g, int& ix, int& iy, int& iz) {
  ix = (int)(h % g.nxh);
  long long r = h / g.nxh;
  iy = (int)(r % g.nx[1]);
  iz = (int)(r / g.nx[1]);
}

// signed frequency index of the reference convention (device_array_utils.cu:67-72)
__host__ __device__ __forceinline__ int sfreq(int n, int N) {
  return ((float)n < (float)N / 2.0f) ? n : n - N;
}

__device__ double k2_fp64(long long h, const Geom& g, int D) {
  int n[3];
  half_index(h, g, n[0], n[1], n[2]);
  double k2 = 0.0;
  for (int d = 0; d < D; d++) {
    const double kd = 2.0 * kPi * (double)sfreq(n[d], g.nx[d]) / (double)g.L[d];
    k2 += kd * kd;
  }
  return k2;
}

__device__ float k2_ref(long long h, const Geom& g, int D) {
  int n[3];
  half_index(h, g, n[0], n[1], n[2]);
  float k2 = 0.0f;
  for (int d = 0; d < D; d++) {
    float kd;
    if ((float)n[d] < (float)g.nx[d] / 2.0f) kd = kRefPI2 * (float)n[d] / g.L[d];
    else kd = kRefPI2 * (float)(n[d] - g.nx[d]) / g.L[d];
    k2 += kd * kd;
  }
  return k2;
}

struct StyleParams {
  int kind;
  double A, sig2, R;
  float Af, sig2f, Rf;
};

// u(k) of one FFT style in FP64
__device__ double u_fp64(const StyleParams& s, double k2) {
  const double k = sqrt(k2);
  const double vp = 4.0 * kPi * s.R * s.R * s.R / 3.0;
  if (s.kind == TILD_STYLE_GAUSSIAN) return s.A * exp(-k2 * s.sig2 / 2.0);
  if (s.kind == TILD_STYLE_ERF) {
    if (k2 == 0.0) return s.A * vp * vp;
    const double t = 4.0 * kPi * (sin(s.R * k) - s.R * k * cos(s.R * k)) / (k2 * k);
    return s.A * exp(-k2 * s.sig2 * 0.5) * t * t;
  }
  if (k2 == 0.0) return s.A * vp;
  return s.A * exp(-k2 * s.sig2 * 0.5) * 4.0 * kPi * (sin(s.R * k) - s.R * k * cos(s.R * k)) / (k2 * k);
}

// u(k) of one FFT style with the reference FP32 expressions
__device__ float u_ref(const StyleParams& s, float k2) {
  const float k = sqrtf(k2);
  const float Ao = s.Af, Rp = s.Rf, sigma2 = s.sig2f;
  if (s.kind == TILD_STYLE_GAUSSIAN) return Ao * expf(-k2 * sigma2 / 2.0f);
  if (s.kind == TILD_STYLE_ERF) {
    if (k2 == 0) return Ao * kRefPI4 * Rp * Rp * Rp / 3 * kRefPI4 * Rp * Rp * Rp / 3;
    const float temp = kRefPI4 * (sinf(Rp * k) - Rp * k * cosf(Rp * k)) / (k2 * k);
    return Ao * expf(-k2 * sigma2 * 0.5f) * temp * temp;
  }
  if (k2 == 0) return Ao * kRefPI4 * Rp * Rp * Rp / 3;
  return Ao * expf(-k2 * sigma2 * 0.5f) * kRefPI4 * (sinf(Rp * k) - Rp * k * cosf(Rp * k)) / (k2 * k);
}

__global__ void k_style_table(float* utab, double* ufull, StyleParams s, Geom g, int D, int ref, double invM) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= g.Mh) return;
  double u;
  if (ref) u = (double)u_ref(s, k2_ref(h, g, D));
  else u = u_fp64(s, k2_fp64(h, g, D));
  utab[h] = (float)(u * invM);
  ufull[h] = u;
}

// charge multiplier: psi_k = 4 pi lB rho_k / (M k^2) e^{-k^2/(2a^2)} (d_prepareElectrostaticPotential,
// device_array_utils.cu:199-220) and E_k = -i k psi_k e^{-k^2/(2a^2)} (:225-241): the force path
// applies the smearing exponential twice.
__global__ void k_charge_table(float* ctab, Geom g, int D, double lB, double a, int ref, double invM) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= g.Mh) return;
  if (ref) {
    const float k2 = k2_ref(h, g, D);
    const float ls = (float)a;
    float v = 0.f;
    if (k2 != 0) {
      const float e = expf(-1 * k2 / (2 * ls * ls));
      v = (4 * kRefPI * (float)lB) / k2 * e * e;
    }
    ctab[h] = (float)((double)v * invM);
  } else {
    const double k2 = k2_fp64(h, g, D);
    double v = 0.0;
    if (k2 != 0.0) v = 4.0 * kPi * lB / k2 * exp(-k2 / (a * a));
    ctab[h] = (float)(v * invM);
  }
}

// F_beta(k) = -i kd_beta u(k) on the half spectrum, Nyquist derivative set to zero: its C2R
// equals Re of the reference's full C2C inverse of f_k (the Nyquist plane of the derivative
// direction only contributes imaginary values there).
__global__ void k_force_kernel(cufftDoubleComplex* out, const double* ufull, Geom g, int D, int beta) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= g.Mh) return;
  int n[3];
  half_index(h, g, n[0], n[1], n[2]);
  const int N = g.nx[beta];
  double kd = 0.0;
  if (!((N % 2 == 0) && n[beta] == N / 2)) kd = 2.0 * kPi * (double)sfreq(n[beta], N) / (double)g.L[beta];
  out[h].x = 0.0;
  out[h].y = -kd * ufull[h];
}

// vr(r) = dr_alpha(r) * f_beta(r) with dr the minimum image of the grid point from the origin
// evaluated in FP32 as d_initVirial does (device_array_utils.cu:456-494).
__global__ void k_virial_real(double* vr, const double* fbeta, Geom g, int D, int alpha) {
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= g.M) return;
  int nn[3] = {0, 0, 0};
  long long r = id;
  nn[0] = (int)(r % g.nx[0]);
  r /= g.nx[0];
  if (D == 3) { nn[1] = (int)(r % g.nx[1]); nn[2] = (int)(r / g.nx[1]); }
  else nn[1] = (int)r;
  float ri = (float)nn[alpha] * g.dx[alpha];
  float dr = ri - 0.0f;
  if (dr > g.Lh[alpha]) dr -= g.L[alpha];
  else if (dr < -g.Lh[alpha]) dr += g.L[alpha];
  vr[id] = (double)dr * fbeta[id];
}

__global__ void k_store_virk(cufftComplex* dst, const cufftDoubleComplex* src, long long Mh, double scale) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= Mh) return;
  dst[h].x = (float)(src[h].x * scale);
  dst[h].y = (float)(src[h].y * scale);
}

// init_device_fieldphase (pair_style_fieldphases.cu:101-185): static field f_r = A grad w.
__global__ void k_fieldphase(float* fr, Geom g, int D, double A, int phase, int dir, int nper, int ref) {
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= g.M) return;
  int nn[3] = {0, 0, 0};
  long long rr = id;
  nn[0] = (int)(rr % g.nx[0]);
  rr /= g.nx[0];
  if (D == 3) { nn[1] = (int)(rr % g.nx[1]); nn[2] = (int)(rr / g.nx[1]); }
  else nn[1] = (int)rr;
  double r[3] = {0, 0, 0};
  for (int d = 0; d < D; d++) r[d] = (double)nn[d] * (double)g.dx[d];
  double f[3] = {0, 0, 0};
  if (phase == 0) {
    const double a = 2.0 * kPi * nper / (double)g.L[dir];
    f[dir] = A * a * cos(a * r[dir]);
  } else if (phase == 2) {
    int d1 = 0, d2 = 1;
    if (dir == d1) d1 = 2;
    else if (dir == d2) d2 = 2;
    const double a1 = 2.0 * kPi * nper / (double)g.L[d1], a2 = 2.0 * kPi * nper / (double)g.L[d2];
    f[d1] = A * a1 * sin(a1 * r[d1]) * cos(a2 * r[d2]);
    f[d2] = A * a2 * sin(a2 * r[d2]) * cos(a1 * r[d1]);
  } else if (phase == 3 && D == 3) {
    double ar[3], c[3], s[3];
    for (int j = 0; j < 3; j++) {
      ar[j] = 2.0 * kPi * nper / (double)g.L[j];
      c[j] = cos(ar[j] * r[j]);
      s[j] = sin(ar[j] * r[j]);
    }
    const double e = s[0] * c[1] + s[1] * c[2] + s[2] * c[0];
    f[0] = -A * e * ar[0] * (c[0] * c[1] - s[2] * s[0]);
    f[1] = -A * e * ar[1] * (c[1] * c[2] - s[0] * s[1]);
    f[2] = -A * e * ar[2] * (c[2] * c[0] - s[1] * s[2]);
  }
  (void)ref;
  for (int d = 0; d < D; d++) fr[(long long)d * g.M + id] = (float)f[d];
}

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

int tild_build_tables(tild_ctx* c, int si) {
  SysHost& h = c->sys[si];
  const Geom& g = h.g;
  const int D = h.D;
  const double invM = 1.0 / (double)g.M;
  const int ref = h.cfg.table_mode == TILD_TABLES_REF_FP32;
  cudaStream_t st = c->stream;

  // per-axis k values: kk for k^2 (reference convention), kd for derivatives (Nyquist = 0)
  {
    std::vector<float> kk(g.nx[0] + g.nx[1] + g.nx[2]), kd(kk.size());
    int off = 0;
    for (int d = 0; d < 3; d++) {
      for (int n = 0; n < g.nx[d]; n++) {
        double k = 0.0;
        if (d < D) k = 2.0 * kPi * (double)sfreq(n, g.nx[d]) / (double)g.L[d];
        kk[off + n] = (float)k;
        kd[off + n] = ((g.nx[d] % 2 == 0) && n == g.nx[d] / 2) ? 0.f : (float)k;
      }
      off += g.nx[d];
    }
    if (tild_check(c, cudaMemcpyAsync(c->kk + h.kd0, kk.data(), kk.size() * 4, cudaMemcpyHostToDevice, st), "copy k")) return TILD_ERR_CUDA;
    if (tild_check(c, cudaMemcpyAsync(c->kd + h.kd0, kd.data(), kd.size() * 4, cudaMemcpyHostToDevice, st), "copy kd")) return TILD_ERR_CUDA;
    if (tild_check(c, cudaStreamSynchronize(st), "sync k")) return TILD_ERR_CUDA;
  }

  const int nfft = (int)h.fft_cfg.size();
  // per-direction real slabs start on 16-byte boundaries (cuFFT rejects a misaligned output)
  const long long Mpad = (g.M + 1) / 2 * 2;
  int rc = TILD_OK;
  cufftHandle pz2d = 0, pd2z = 0;
  if (nfft > 0) {
    rc = tild_table_scratch(c);
    if (rc) return rc;
    rc = tild_table_plans(c, g, D, &pz2d, &pd2z);
    if (rc) return rc;
  }
  double* ufull = c->tab_ufull;
  cufftDoubleComplex* zbuf = c->tab_z;
  cufftDoubleComplex* zbuf2 = c->tab_z2;
  double* freal = c->tab_freal;
  double* vr = c->tab_vr;
  SysDev& hd = c->h_sys[si];
  for (int s = 0; s < nfft && rc == TILD_OK; s++) {
    const tild_pair_style& ps = h.cfg.styles[h.fft_cfg[s]];
    StyleParams sp;
    sp.kind = ps.style;
    sp.A = ps.prefactor;
    sp.sig2 = (double)ps.sigma * (double)ps.sigma;
    sp.R = ps.rp;
    sp.Af = ps.prefactor;
    sp.sig2f = (float)sp.sig2;
    sp.Rf = ps.rp;
    k_style_table<<<nblk(g.Mh, 256), 256, 0, st>>>(c->utab + h.utab0 + (long long)s * g.Mh, ufull, sp, g, D, ref, invM);
    c->launches++;
    double u0 = 0.0;
    if (tild_check(c, cudaMemcpyAsync(&u0, ufull, sizeof(double), cudaMemcpyDeviceToHost, st), "u0") ||
        tild_check(c, cudaStreamSynchronize(st), "sync u0")) { rc = TILD_ERR_CUDA; break; }
    hd.suk0[s] = (float)u0;
    // real-space force table f_beta(r), unnormalised inverse transform
    for (int beta = 0; beta < D && rc == TILD_OK; beta++) {
      k_force_kernel<<<nblk(g.Mh, 256), 256, 0, st>>>(zbuf, ufull, g, D, beta);
      c->launches++;
      if (tild_check_fft(c, cufftExecZ2D(pz2d, zbuf, freal + (long long)beta * Mpad), "exec z2d")) rc = TILD_ERR_CUDA;
    }
    // virial kernels: FFT(dr_alpha f_beta) / M (InitializeVirial), times the 1/M that
    // CalcVirial applies to rho_k (pair_style.cu:277-279), stored on the half spectrum.
    const int ab[6][2] = {{0, 0}, {1, 1}, {2, 2}, {1, 0}, {2, 0}, {2, 1}};   // (alpha, beta)
    const int ab2[3][2] = {{0, 0}, {1, 1}, {1, 0}};
    for (int j = 0; j < h.nP && rc == TILD_OK; j++) {
      const int alpha = (D == 3) ? ab[j][0] : ab2[j][0];
      const int beta = (D == 3) ? ab[j][1] : ab2[j][1];
      k_virial_real<<<nblk(g.M, 256), 256, 0, st>>>(vr, freal + (long long)beta * Mpad, g, D, alpha);
      c->launches++;
      if (tild_check_fft(c, cufftExecD2Z(pd2z, vr, zbuf2), "exec d2z")) { rc = TILD_ERR_CUDA; break; }
      k_store_virk<<<nblk(g.Mh, 256), 256, 0, st>>>(c->virk + h.virk0 + ((long long)s * h.nP + j) * g.Mh, zbuf2, g.Mh,
                                                    invM * invM);
      c->launches++;
    }
  }
  if (rc == TILD_OK && h.C) {
    k_charge_table<<<nblk(g.Mh, 256), 256, 0, st>>>(c->ctab + h.ctab0, g, D, h.cfg.bjerrum, h.cfg.smearing, ref, invM);
    c->launches++;
  }
  for (const FieldK& fk : c->fields) {
    if (fk.sys != si || rc != TILD_OK) continue;
    const tild_pair_style& ps = h.cfg.styles[fk.cfg_index];
    k_fieldphase<<<nblk(g.M, 256), 256, 0, st>>>(c->frfield + fk.fr0, g, D, ps.prefactor, ps.phase, ps.dir,
                                                 ps.n_periods, ref);
    c->launches++;
  }
  if (rc == TILD_OK && tild_check(c, cudaStreamSynchronize(st), "table build")) rc = TILD_ERR_CUDA;
  return rc;
}

// Scratch of the FP64 table builds, sized once for the largest grid of the engine and kept, so
// that reloading a system (tild_batch_load) allocates nothing.
int tild_table_scratch(tild_ctx* c) {
  if (c->tab_ufull) return TILD_OK;
  long long M = 1, Mh = 1;
  int D = 3;
  for (const SysHost& h : c->sys) {
    M = std::max(M, h.g.M);
    Mh = std::max(Mh, h.g.Mh);
    D = h.D;
  }
  const long long Mpad = (M + 1) / 2 * 2;
  if (tild_check(c, cudaMalloc(&c->tab_ufull, sizeof(double) * Mh), "alloc table scratch") ||
      tild_check(c, cudaMalloc(&c->tab_z, sizeof(cufftDoubleComplex) * Mh), "alloc table scratch") ||
      tild_check(c, cudaMalloc(&c->tab_z2, sizeof(cufftDoubleComplex) * Mh), "alloc table scratch") ||
      tild_check(c, cudaMalloc(&c->tab_freal, sizeof(double) * Mpad * D), "alloc table scratch") ||
      tild_check(c, cudaMalloc(&c->tab_vr, sizeof(double) * M), "alloc table scratch"))
    return TILD_ERR_OOM;
  c->tab_M = M;
  return TILD_OK;
}

// Z2D / D2Z plans of one grid shape, made once per shape and kept for the engine's lifetime.
int tild_table_plans(tild_ctx* c, const Geom& g, int D, cufftHandle* z2d, cufftHandle* d2z) {
  for (const auto& tp : c->tab_plans)
    if (tp.nx[0] == g.nx[0] && tp.nx[1] == g.nx[1] && tp.nx[2] == g.nx[2]) {
      *z2d = tp.z2d;
      *d2z = tp.d2z;
      return TILD_OK;
    }
  int n[3];
  if (D == 3) { n[0] = g.nx[2]; n[1] = g.nx[1]; n[2] = g.nx[0]; }
  else { n[0] = g.nx[1]; n[1] = g.nx[0]; }
  tild_ctx::TablePlan tp;
  for (int q = 0; q < 3; q++) tp.nx[q] = g.nx[q];
  tp.z2d = tp.d2z = 0;
  if (tild_check_fft(c, cufftPlanMany(&tp.z2d, D, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, 1), "plan z2d"))
    return TILD_ERR_CUDA;
  if (tild_check_fft(c, cufftPlanMany(&tp.d2z, D, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 1), "plan d2z")) {
    cufftDestroy(tp.z2d);
    return TILD_ERR_CUDA;
  }
  if (tild_check_fft(c, cufftSetStream(tp.z2d, c->stream), "stream z2d") ||
      tild_check_fft(c, cufftSetStream(tp.d2z, c->stream), "stream d2z")) {
    cufftDestroy(tp.z2d);
    cufftDestroy(tp.d2z);
    return TILD_ERR_CUDA;
  }
  c->tab_plans.push_back(tp);
  *z2d = tp.z2d;
  *d2z = tp.d2z;
  return TILD_OK;
}

void tild_tables_free(tild_ctx* c) {
  for (auto& tp : c->tab_plans) {
    cufftDestroy(tp.z2d);
    cufftDestroy(tp.d2z);
  }
  c->tab_plans.clear();
  void* ptrs[] = {c->tab_ufull, c->tab_z, c->tab_z2, c->tab_freal, c->tab_vr};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  c->tab_ufull = nullptr;
  c->tab_z = c->tab_z2 = nullptr;
  c->tab_freal = c->tab_vr = nullptr;
}
