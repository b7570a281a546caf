/*
 * tild_oracle.c — FP64 CPU restatement of gpu-tild's per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, __graft_entry__.smoke() and
 * the cpu_baseline / reference legs of bench.py call it to produce the numbers the CUDA
 * library (libtild.so) is compared against.  Nothing in the product links or calls it.
 *
 * It follows the reference algorithm literally rather than the CUDA library's reformulation:
 *  - full complex-to-complex FFTs, one forward per density and Dim inverse transforms per
 *    pair style and side (pair_style.cu:119-235), with the reference's k vector convention
 *    (device_array_utils.cu:60-82, Nyquist bin mapped negative);
 *  - grid forces accumulated as rho_I * Re(IFFT(f_k rho_J / M)) (device_array_utils.cu:298-312,
 *    362-372) and divided by rho again in the gather with the rho > 0 guard
 *    (device_grid_utils.cu:424-452);
 *  - energies and virials in real space (pair_style.cu:204-276), bonds on the host
 *    (bonds.cu:3-52), electrostatics as sum psi*rho_c (calc_properties.cu:106-116).
 * Arithmetic is FP64 except the quantities whose FP32 value decides an integer (grid index
 * of a bead, cell index, minimum-image comparisons), which are evaluated in FP32 exactly as
 * the reference does so that stencil indices and cells match bit for bit.
 *
 * The FFT is a self-contained recursive mixed-radix Cooley-Tukey transform (decimation in
 * time, radix = each prime factor, direct DFT for the prime butterflies).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/tild.h"

typedef struct { double re, im; } cpx;

static inline cpx cmul(cpx a, cpx b) { cpx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }

/* ------------------------------------------------------------------------------------- */
/* FFT                                                                                    */
/* ------------------------------------------------------------------------------------- */
typedef struct {
  int n, nf, fac[64], maxp;
  cpx* tw; /* tw[j] = exp(-2 pi i j / n) */
} fft1;

static void fft1_init(fft1* p, int n) {
  p->n = n; p->nf = 0; p->maxp = 1;
  int m = n;
  for (int f = 2; m > 1;) {
    if (m % f == 0) { p->fac[p->nf++] = f; if (f > p->maxp) p->maxp = f; m /= f; }
    else { f = (f == 2) ? 3 : f + 2; if (f * f > m && m > 1) { f = m; } }
  }
  p->tw = (cpx*)malloc(sizeof(cpx) * (size_t)n);
  for (int j = 0; j < n; j++) {
    double a = -2.0 * M_PI * (double)j / (double)n;
    p->tw[j].re = cos(a); p->tw[j].im = sin(a);
  }
}
static void fft1_free(fft1* p) { free(p->tw); p->tw = NULL; }

/* out[k] = sum_j in[j*is] w^{jk}, length n = product of fac[..]; twstep = N/n. */
static void fft_rec(const cpx* in, int is, cpx* out, int n, const int* fac, const fft1* P,
                    int twstep, int sign, cpx* scratch) {
  const int N = P->n;
  const int p = fac[0], m = n / p;
  if (m == 1) {
    for (int k = 0; k < p; k++) {
      cpx s = {0.0, 0.0};
      for (int r = 0; r < p; r++) {
        cpx w = P->tw[(int)(((long)r * k * twstep) % N)];
        if (sign > 0) w.im = -w.im;
        cpx t = cmul(in[(long)r * is], w);
        s.re += t.re; s.im += t.im;
      }
      out[k] = s;
    }
    return;
  }
  for (int r = 0; r < p; r++) fft_rec(in + (long)r * is, is * p, out + (long)r * m, m, fac + 1, P, twstep * p, sign, scratch);
  for (int k = 0; k < m; k++) {
    for (int r = 0; r < p; r++) {
      cpx w = P->tw[(int)(((long)r * k * twstep) % N)];
      if (sign > 0) w.im = -w.im;
      scratch[r] = cmul(out[(long)r * m + k], w);
    }
    for (int q = 0; q < p; q++) {
      cpx s = {0.0, 0.0};
      for (int r = 0; r < p; r++) {
        cpx w = P->tw[(int)(((long)r * q * m * twstep) % N)];
        if (sign > 0) w.im = -w.im;
        cpx t = cmul(scratch[r], w);
        s.re += t.re; s.im += t.im;
      }
      scratch[p + q] = s;
    }
    for (int q = 0; q < p; q++) out[(long)q * m + k] = scratch[p + q];
  }
}

/* 1D transform of a strided line, in place. buf needs 2n + 2*maxp entries. */
static void fft_line(const fft1* P, cpx* data, long stride, int sign, cpx* buf) {
  const int n = P->n;
  if (n == 1) return;
  cpx* a = buf; cpx* b = buf + n; cpx* s = buf + 2 * n;
  for (int j = 0; j < n; j++) a[j] = data[(long)j * stride];
  fft_rec(a, 1, b, n, P->fac, P, 1, sign, s);
  for (int j = 0; j < n; j++) data[(long)j * stride] = b[j];
}

typedef struct { int dim; int nx[3]; fft1 p[3]; int maxn, maxp; } fftnd;

static void fftnd_init(fftnd* F, int dim, const int* nx) {
  F->dim = dim; F->maxn = 1; F->maxp = 1;
  for (int d = 0; d < 3; d++) F->nx[d] = (d < dim) ? nx[d] : 1;
  for (int d = 0; d < dim; d++) {
    fft1_init(&F->p[d], nx[d]);
    if (nx[d] > F->maxn) F->maxn = nx[d];
    if (F->p[d].maxp > F->maxp) F->maxp = F->p[d].maxp;
  }
}
static void fftnd_free(fftnd* F) { for (int d = 0; d < F->dim; d++) fft1_free(&F->p[d]); }

/* Unnormalised transform of data laid out x fastest: idx = x + (y + z*Ny)*Nx.
 * sign = -1 forward (CUFFT_FORWARD), +1 inverse (CUFFT_INVERSE). */
static void fftnd_exec(const fftnd* F, cpx* data, int sign) {
  const long Nx = F->nx[0], Ny = F->nx[1], Nz = F->nx[2];
  const long M = Nx * Ny * Nz;
  const int bufn = 2 * F->maxn + 2 * F->maxp + 8;
  for (int axis = 0; axis < F->dim; axis++) {
    long nlines, stride;
    if (axis == 0) { nlines = M / Nx; stride = 1; }
    else if (axis == 1) { nlines = M / Ny; stride = Nx; }
    else { nlines = M / Nz; stride = Nx * Ny; }
#pragma omp parallel
    {
      cpx* buf = (cpx*)malloc(sizeof(cpx) * (size_t)bufn);
#pragma omp for schedule(static)
      for (long l = 0; l < nlines; l++) {
        long base;
        if (axis == 0) base = l * Nx;
        else if (axis == 1) { long x = l % Nx, z = l / Nx; base = x + z * Nx * Ny; }
        else base = l;
        fft_line(&F->p[axis], data + base, stride, sign, buf);
      }
      free(buf);
    }
  }
}

/* Exported for the FFT self-test against numpy. data: interleaved complex, in place. */
int orc_fft(int dim, const int* nx, double* data, int sign) {
  fftnd F; fftnd_init(&F, dim, nx);
  fftnd_exec(&F, (cpx*)data, sign);
  fftnd_free(&F);
  return 0;
}

/* ------------------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and the normal draws used for noise.  */
/* The CUDA library derives its noise from the same counter layout.                      */
/* ------------------------------------------------------------------------------------- */
static void philox4x32_10(uint32_t ctr[4], const uint32_t key_in[2]) {
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int round = 0; round < 10; round++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ ctr[1] ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ ctr[3] ^ k1;
    uint32_t n3 = lo0;
    ctr[0] = n0; ctr[1] = n1; ctr[2] = n2; ctr[3] = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
}

/* Three standard normals for (seed, bead, step, integrator): Box-Muller on 24-bit uniforms. */
static void noise3(uint64_t seed, uint32_t bead, int64_t step, uint32_t integ, double out[3]) {
  uint32_t ctr[4] = {(uint32_t)step, (uint32_t)((uint64_t)step >> 32), integ, (uint32_t)(seed >> 32)};
  uint32_t key[2] = {bead, (uint32_t)seed};
  philox4x32_10(ctr, key);
  /* 24-bit uniforms; the odd numerator keeps u0, u2 in (0,1) and exactly representable in
   * FP32, so the CUDA side draws bit-identical uniforms */
  double u0 = (double)((ctr[0] >> 8) | 1u) * (1.0 / 16777216.0);
  double u1 = (double)(ctr[1] >> 8) * (1.0 / 16777216.0);
  double u2 = (double)((ctr[2] >> 8) | 1u) * (1.0 / 16777216.0);
  double u3 = (double)(ctr[3] >> 8) * (1.0 / 16777216.0);
  double r0 = sqrt(-2.0 * log(u0)), r1 = sqrt(-2.0 * log(u2));
  out[0] = r0 * cos(2.0 * M_PI * u1);
  out[1] = r0 * sin(2.0 * M_PI * u1);
  out[2] = r1 * cos(2.0 * M_PI * u3);
}

/* Exported so tests can compare the two implementations of the noise stream directly. */
int orc_noise3(uint64_t seed, uint32_t bead, int64_t step, uint32_t integ, double* out) {
  noise3(seed, bead, step, integ, out);
  return 0;
}

/* ------------------------------------------------------------------------------------- */
/* System                                                                                 */
/* ------------------------------------------------------------------------------------- */
typedef struct orc_sys {
  tild_config cfg;
  int D, T, ns, p, S, nP, M, C; /* C = 1 if charges */
  int Nx[3];
  float L[3], Lh[3], dx[3];  /* FP32 as in the reference (config_utils.cu:35-48, initialize.cu:36) */
  double gvol, dV, V;
  fftnd F;
  /* topology */
  int32_t* tp; float* q; int32_t* nb; int32_t* bto; int32_t* bty;
  /* per style k-space tables (full spectrum) */
  double* uk[TILD_MAX_STYLES];        /* u_k real part (imaginary part is zero) */
  double* uk0[TILD_MAX_STYLES];       /* scalar u_k[0] at setup, for ramps */
  cpx* virk[TILD_MAX_STYLES];         /* [nP][M] */
  double* fr[TILD_MAX_STYLES];        /* fieldphase real-space field [M*D] */
  double* kvec;                       /* [M*D] reference k vectors */
  double* k2;                         /* [M] */
  /* state of the last force evaluation */
  double* rho;                        /* [(T+C)*M] */
  cpx* rhok;                          /* [(T+C)*M] FFT of each density */
  double* gridF;                      /* [D][T][M] grid forces */
  double* Efield;                     /* [D][M] electric field */
  double* psi;                        /* [M] electrostatic potential */
  int have_forces;
  int64_t forces_step;
  cpx* work; cpx* work2;
} orc_sys;

static void stack_r(const orc_sys* s, int id, int nn[3]) {
  /* reference unstack (array_utils.cu:62-81) */
  if (s->D == 2) { nn[1] = id / s->Nx[0]; nn[0] = id - nn[1] * s->Nx[0]; nn[2] = 0; }
  else { nn[2] = id / s->Nx[1] / s->Nx[0]; nn[1] = id / s->Nx[0] - nn[2] * s->Nx[1];
         nn[0] = id - (nn[1] + nn[2] * s->Nx[1]) * s->Nx[0]; }
}

/* Ramp multiplier of style i for a force evaluation at step `step` (pair_style.cu:347-367:
 * after each update u_k(0) equals the ramped prefactor). */
static double ramp_ratio(const orc_sys* s, int i, int64_t step) {
  const tild_pair_style* ps = &s->cfg.styles[i];
  if (!ps->ramp || step < 2 || s->cfg.max_steps <= 0) return 1.0;
  double Ai = ps->prefactor, Af = ps->final_prefactor;
  double target = Ai + (Ai - Af) * (double)step / (double)s->cfg.max_steps;
  return target / s->uk0[i][0];
}

static int style_rank(int st) { /* evaluation order of forces.cu:106-129 */
  switch (st) { case TILD_STYLE_GAUSSIAN: return 0; case TILD_STYLE_ERF: return 1;
                case TILD_STYLE_FIELDPHASE: return 2; default: return 3; }
}

static void build_tables(orc_sys* s) {
  const int M = s->M, D = s->D;
  s->kvec = (double*)malloc(sizeof(double) * (size_t)M * D);
  s->k2 = (double*)malloc(sizeof(double) * (size_t)M);
  for (int id = 0; id < M; id++) {
    int nn[3]; stack_r(s, id, nn);
    double k2 = 0.0;
    for (int d = 0; d < D; d++) {
      /* device_array_utils.cu:67-72: n < N/2 -> positive, else n - N (Nyquist negative) */
      double kd = ((float)nn[d] < (float)s->Nx[d] / 2.0) ? 2.0 * M_PI * nn[d] / (double)s->L[d]
                                                           : 2.0 * M_PI * (nn[d] - s->Nx[d]) / (double)s->L[d];
      s->kvec[(size_t)id * D + d] = kd; k2 += kd * kd;
    }
    s->k2[id] = k2;
  }
  cpx* f = (cpx*)malloc(sizeof(cpx) * (size_t)M);
  double* freal = (double*)malloc(sizeof(double) * (size_t)M * D);
  double* vr = (double*)malloc(sizeof(double) * (size_t)M);
  for (int i = 0; i < s->cfg.n_styles; i++) {
    const tild_pair_style* ps = &s->cfg.styles[i];
    s->uk0[i] = (double*)malloc(sizeof(double));
    if (ps->style == TILD_STYLE_FIELDPHASE) {
      /* init_device_fieldphase, pair_style_fieldphases.cu:101-185 */
      s->fr[i] = (double*)calloc((size_t)M * D, sizeof(double));
      s->uk0[i][0] = 1.0;
      double A = ps->prefactor;
      for (int id = 0; id < M; id++) {
        int nn[3]; stack_r(s, id, nn);
        double r[3] = {0, 0, 0};
        for (int d = 0; d < D; d++) r[d] = (double)nn[d] * (double)s->dx[d];
        double* fo = s->fr[i] + (size_t)id * D;
        if (ps->phase == 0) {
          double a = 2.0 * M_PI * ps->n_periods / (double)s->L[ps->dir];
          for (int j = 0; j < D; j++) fo[j] = (j == ps->dir) ? A * a * cos(a * r[ps->dir]) : 0.0;
        } else if (ps->phase == 2) {
          int d1 = 0, d2 = 1;
          if (ps->dir == d1) d1 = 2; else if (ps->dir == d2) d2 = 2;
          double a1 = 2.0 * M_PI * ps->n_periods / (double)s->L[d1];
          double a2 = 2.0 * M_PI * ps->n_periods / (double)s->L[d2];
          if (D == 3) fo[ps->dir] = 0.0;
          fo[d1] = A * a1 * sin(a1 * r[d1]) * cos(a2 * r[d2]);
          fo[d2] = A * a2 * sin(a2 * r[d2]) * cos(a1 * r[d1]);
        } else if (ps->phase == 3 && D == 3) {
          double ar[3], c[3], sn[3];
          for (int j = 0; j < 3; j++) { ar[j] = 2.0 * M_PI * ps->n_periods / (double)s->L[j];
                                        c[j] = cos(ar[j] * r[j]); sn[j] = sin(ar[j] * r[j]); }
          double e = sn[0] * c[1] + sn[1] * c[2] + sn[2] * c[0];
          fo[0] = -A * e * ar[0] * (c[0] * c[1] - sn[2] * sn[0]);
          fo[1] = -A * e * ar[1] * (c[1] * c[2] - sn[0] * sn[1]);
          fo[2] = -A * e * ar[2] * (c[2] * c[0] - sn[1] * sn[2]);
        }
      }
      continue;
    }
    s->uk[i] = (double*)malloc(sizeof(double) * (size_t)M);
    double A = ps->prefactor, sig2 = (double)ps->sigma * (double)ps->sigma, R = ps->rp;
    double vp = 4.0 * M_PI * R * R * R / 3.0;
    for (int id = 0; id < M; id++) {
      double k2 = s->k2[id], k = sqrt(k2), u;
      if (ps->style == TILD_STYLE_GAUSSIAN) u = A * exp(-k2 * sig2 / 2.0);
      else if (ps->style == TILD_STYLE_ERF) {
        if (k2 == 0.0) u = A * vp * vp;
        else { double t = 4.0 * M_PI * (sin(R * k) - R * k * cos(R * k)) / (k2 * k);
               u = A * exp(-k2 * sig2 * 0.5) * t * t; }
      } else {
        if (k2 == 0.0) u = A * vp;
        else u = A * exp(-k2 * sig2 * 0.5) * 4.0 * M_PI * (sin(R * k) - R * k * cos(R * k)) / (k2 * k);
      }
      s->uk[i][id] = u;
    }
    s->uk0[i][0] = s->uk[i][0];
    /* real-space force table: unnormalised IFFT of f_k = -i k u_k (pair_style_gaussian.cu:36-41) */
    for (int d = 0; d < D; d++) {
      for (int id = 0; id < M; id++) { f[id].re = 0.0; f[id].im = -s->kvec[(size_t)id * D + d] * s->uk[i][id]; }
      fftnd_exec(&s->F, f, +1);
      for (int id = 0; id < M; id++) freal[(size_t)id * D + d] = f[id].re;
    }
    /* virial tables, d_initVirial (device_array_utils.cu:456-494) + InitializeVirial */
    s->virk[i] = (cpx*)malloc(sizeof(cpx) * (size_t)M * s->nP);
    for (int j = 0; j < s->nP; j++) {
      for (int id = 0; id < M; id++) {
        int nn[3]; stack_r(s, id, nn);
        float drf[3] = {0, 0, 0};
        for (int d = 0; d < D; d++) {
          float ri = (float)nn[d] * s->dx[d];
          float dr = ri - 0.0f;
          if (dr > s->Lh[d]) dr -= s->L[d]; else if (dr < -s->Lh[d]) dr += s->L[d];
          drf[d] = dr;
        }
        const double* fo = freal + (size_t)id * D;
        double v;
        if (j < D) v = (double)drf[j] * fo[j];
        else if (D == 2) v = (double)drf[1] * fo[0];          /* xy */
        else if (j == 3) v = (double)drf[1] * fo[0];          /* xy */
        else if (j == 4) v = (double)drf[2] * fo[0];          /* xz */
        else v = (double)drf[2] * fo[1];                      /* yz */
        f[id].re = v; f[id].im = 0.0;
      }
      fftnd_exec(&s->F, f, -1);
      for (int id = 0; id < M; id++) { s->virk[i][(size_t)j * M + id].re = f[id].re / M;
                                       s->virk[i][(size_t)j * M + id].im = f[id].im / M; }
    }
  }
  free(f); free(freal); free(vr);
}

int orc_create(const tild_config* cfg, orc_sys** out) {
  if (!cfg || !out) return TILD_ERR_BAD_INPUT;
  if (cfg->dim != 2 && cfg->dim != 3) return TILD_ERR_BAD_INPUT;
  if (cfg->pmeorder < 0 || cfg->pmeorder > 4) return TILD_ERR_BAD_INPUT;
  orc_sys* s = (orc_sys*)calloc(1, sizeof(orc_sys));
  s->cfg = *cfg;
  s->D = cfg->dim; s->T = cfg->ntypes; s->ns = cfg->ns; s->p = cfg->pmeorder;
  s->C = cfg->do_charges ? 1 : 0;
  s->nP = (s->D == 2) ? 3 : 6;
  s->M = 1; s->S = 1;
  float gv = 1.0f;
  for (int d = 0; d < 3; d++) { s->Nx[d] = (d < s->D) ? cfg->nx[d] : 1; }
  for (int d = 0; d < s->D; d++) {
    s->L[d] = cfg->box[d]; s->Lh[d] = 0.5f * s->L[d];
    s->dx[d] = s->L[d] / (float)s->Nx[d];
    gv *= s->dx[d];
    s->M *= s->Nx[d]; s->S *= (s->p + 1);
  }
  s->gvol = (double)gv;
  s->dV = 1.0; s->V = 1.0;
  for (int d = 0; d < s->D; d++) { s->dV *= (double)s->dx[d]; s->V *= (double)s->L[d]; }
  fftnd_init(&s->F, s->D, s->Nx);
  build_tables(s);
  const size_t M = (size_t)s->M;
  s->rho = (double*)calloc((size_t)(s->T + s->C) * M, sizeof(double));
  s->rhok = (cpx*)calloc((size_t)(s->T + s->C) * M, sizeof(cpx));
  s->gridF = (double*)calloc((size_t)s->D * s->T * M, sizeof(double));
  s->Efield = (double*)calloc((size_t)s->D * M, sizeof(double));
  s->psi = (double*)calloc(M, sizeof(double));
  s->work = (cpx*)malloc(sizeof(cpx) * M);
  s->work2 = (cpx*)malloc(sizeof(cpx) * M);
  *out = s;
  return TILD_OK;
}

void orc_destroy(orc_sys* s) {
  if (!s) return;
  for (int i = 0; i < s->cfg.n_styles; i++) { free(s->uk[i]); free(s->uk0[i]); free(s->virk[i]); free(s->fr[i]); }
  free(s->kvec); free(s->k2);
  free(s->rho); free(s->rhok); free(s->gridF); free(s->Efield); free(s->psi); free(s->work); free(s->work2);
  free(s->tp); free(s->q); free(s->nb); free(s->bto); free(s->bty);
  fftnd_free(&s->F);
  free(s);
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int orc_set_topology(orc_sys* s, const int32_t* types, const float* charges, const int32_t* nb,
                     const int32_t* bto, const int32_t* bty) {
  const size_t ns = (size_t)s->ns;
  free(s->tp); free(s->q); free(s->nb); free(s->bto); free(s->bty);
  s->tp = (int32_t*)malloc(ns * 4); memcpy(s->tp, types, ns * 4);
  for (size_t i = 0; i < ns; i++) if (types[i] < 0 || types[i] >= s->T) return TILD_ERR_BAD_INPUT;
  s->q = (float*)calloc(ns, 4); if (charges) memcpy(s->q, charges, ns * 4);
  s->nb = (int32_t*)calloc(ns, 4); if (nb) memcpy(s->nb, nb, ns * 4);
  s->bto = (int32_t*)calloc(ns * 3, 4); if (bto) memcpy(s->bto, bto, ns * 12);
  s->bty = (int32_t*)calloc(ns * 3, 4); if (bty) memcpy(s->bty, bty, ns * 12);
  return TILD_OK;
}

/* ---- assignment weights: spline_get_weights (device_grid_utils.cu:3-49), incl. the
 *      order-4 sx3 = sx2*sx2 of line 39 ----------------------------------------------- */
static void weights(double gdx, double H, double* W, int p) {
  double sx = gdx / H, sx2, sx3, sx4;
  if (p == 0) W[0] = 1.0;
  else if (p == 1) { W[0] = 0.5 - sx; W[1] = 0.5 + sx; }
  else if (p == 2) { sx2 = sx * sx; W[0] = 0.125 - 0.5 * sx + 0.5 * sx2; W[1] = 0.75 - sx2;
                     W[2] = 0.125 + 0.5 * sx + 0.5 * sx2; }
  else if (p == 3) { sx2 = sx * sx; sx3 = sx2 * sx;
    W[0] = (1.0 - 6.0 * sx + 12.0 * sx2 - 8.0 * sx3) / 48.0;
    W[1] = (23.0 - 30.0 * sx - 12.0 * sx2 + 24.0 * sx3) / 48.0;
    W[2] = (23.0 + 30.0 * sx - 12.0 * sx2 - 24.0 * sx3) / 48.0;
    W[3] = (1.0 + 6.0 * sx + 12.0 * sx2 + 8.0 * sx3) / 48.0; }
  else { sx2 = sx * sx; sx3 = sx2 * sx2; sx4 = sx2 * sx2;
    W[0] = (1.0 - 8.0 * sx + 24.0 * sx2 - 32.0 * sx3 + 16.0 * sx4) / 384.0;
    W[1] = (19.0 - 44.0 * sx + 24.0 * sx2 + 16.0 * sx3 - 16.0 * sx4) / 96.0;
    W[2] = (115.0 - 120.0 * sx2 + 48.0 * sx4) / 192.0;
    W[3] = (19.0 + 44.0 * sx + 24.0 * sx2 - 16.0 * sx3 - 16.0 * sx4) / 96.0;
    W[4] = (1.0 + 8.0 * sx + 24.0 * sx2 + 32.0 * sx3 + 16.0 * sx4) / 384.0; }
}

/* Stencil of one bead as d_charge_grid builds it (device_grid_utils.cu:232-343).
 * Returns 0, or -1 if an index falls outside the grid after the reference's single wrap. */
static int bead_stencil(const orc_sys* s, const float* xb, int* inds, double* w) {
  const int D = s->D, p = s->p;
  int g[3] = {0, 0, 0};
  double W[3][6] = {{0}};
  for (int j = 0; j < D; j++) {
    float xj = xb[j], dxj = s->dx[j];
    double gdx;
    if (p % 2 == 0) { g[j] = (int)((xj + 0.5f * dxj) / dxj); gdx = (double)xj - (double)g[j] * (double)dxj; }
    else { g[j] = (int)(xj / dxj); gdx = (double)xj - ((double)g[j] + 0.5) * (double)dxj; }
    weights(gdx, (double)dxj, W[j], p);
  }
  const int sh = p / 2;
  int ct = 0;
  if (D == 2) {
    for (int ix = 0; ix <= p; ix++) {
      int n0 = g[0] + ix - sh; if (n0 < 0) n0 += s->Nx[0]; else if (n0 >= s->Nx[0]) n0 -= s->Nx[0];
      for (int iy = 0; iy <= p; iy++) {
        int n1 = g[1] + iy - sh; if (n1 < 0) n1 += s->Nx[1]; else if (n1 >= s->Nx[1]) n1 -= s->Nx[1];
        if (n0 < 0 || n0 >= s->Nx[0] || n1 < 0 || n1 >= s->Nx[1]) return -1;
        inds[ct] = n1 * s->Nx[0] + n0;
        w[ct] = W[0][ix] * W[1][iy] / s->gvol;
        ct++;
      }
    }
  } else {
    for (int ix = 0; ix <= p; ix++) {
      int n0 = g[0] + ix - sh; if (n0 < 0) n0 += s->Nx[0]; else if (n0 >= s->Nx[0]) n0 -= s->Nx[0];
      for (int iy = 0; iy <= p; iy++) {
        int n1 = g[1] + iy - sh; if (n1 < 0) n1 += s->Nx[1]; else if (n1 >= s->Nx[1]) n1 -= s->Nx[1];
        for (int iz = 0; iz <= p; iz++) {
          int n2 = g[2] + iz - sh; if (n2 < 0) n2 += s->Nx[2]; else if (n2 >= s->Nx[2]) n2 -= s->Nx[2];
          if (n0 < 0 || n0 >= s->Nx[0] || n1 < 0 || n1 >= s->Nx[1] || n2 < 0 || n2 >= s->Nx[2]) return -1;
          inds[ct] = n0 + (n1 + n2 * s->Nx[1]) * s->Nx[0];
          w[ct] = W[0][ix] * W[1][iy] * W[2][iz] / s->gvol;
          ct++;
        }
      }
    }
  }
  return 0;
}

int orc_stencil(orc_sys* s, const float* x, int32_t* inds, double* w) {
  const int S = s->S, D = s->D;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (long i = 0; i < s->ns; i++) {
    int li[128]; double lw[128];
    if (bead_stencil(s, x + i * D, li, lw)) { bad = 1; continue; }
    for (int m = 0; m < S; m++) { if (inds) inds[i * S + m] = li[m]; if (w) w[i * S + m] = lw[m]; }
  }
  return bad ? TILD_ERR_BAD_INPUT : TILD_OK;
}

/* ---- forces(): forces.cu:42-196 ----------------------------------------------------- */
static void fft_real(const orc_sys* s, const double* re, cpx* out, int sign) {
  for (long i = 0; i < s->M; i++) { out[i].re = re[i]; out[i].im = 0.0; }
  fftnd_exec(&s->F, out, sign);
}

int orc_forces(orc_sys* s, const float* x, int64_t step, double* fout, double* rho_out) {
  const int D = s->D, T = s->T, S = s->S;
  const long M = s->M, ns = s->ns;
  if (!s->tp) return TILD_ERR_STATE;
  for (long i = 0; i < ns * D; i++) if (!isfinite(x[i])) return TILD_ERR_NAN;
  memset(s->rho, 0, sizeof(double) * (size_t)(T + s->C) * M);
  memset(s->gridF, 0, sizeof(double) * (size_t)D * T * M);
  int bad = 0;
  /* d_charge_grid / d_charge_grid_charges: accumulate W/gvol (and q W/gvol) */
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (long i = 0; i < ns; i++) {
    int li[128]; double lw[128];
    if (bead_stencil(s, x + i * D, li, lw)) { bad = 1; continue; }
    double* rt = s->rho + (size_t)s->tp[i] * M;
    for (int m = 0; m < S; m++) {
#pragma omp atomic
      rt[li[m]] += lw[m];
      if (s->C) {
#pragma omp atomic
        s->rho[(size_t)T * M + li[m]] += lw[m] * (double)s->q[i];
      }
    }
  }
  if (bad) return TILD_ERR_BAD_INPUT;
  /* FFT of every density (PairStyle::CalcForces transforms rho_J, then rho_I) */
  for (int t = 0; t < T + s->C; t++) fft_real(s, s->rho + (size_t)t * M, s->rhok + (size_t)t * M, -1);
  cpx* tmp = s->work;
  /* pair styles in the reference order: Gaussians, Erfs, FieldPhases, GaussianErfs */
  for (int rank = 0; rank < 4; rank++) {
    for (int i = 0; i < s->cfg.n_styles; i++) {
      const tild_pair_style* ps = &s->cfg.styles[i];
      if (style_rank(ps->style) != rank) continue;
      const int a = ps->type1, b = ps->type2;
      if (ps->style == TILD_STYLE_FIELDPHASE) {
        /* d_prepareFieldForce + d_accumulateGridForce: force_a += rho_a * (rho_a fr),
         * force_b += rho_b * (-rho_b fr) (device_array_utils.cu:410-423, 362-372) */
        for (int d = 0; d < D; d++) {
          double* Fa = s->gridF + ((size_t)d * T + a) * M;
          double* Fb = s->gridF + ((size_t)d * T + b) * M;
          for (long r = 0; r < M; r++) {
            double fr = s->fr[i][(size_t)r * D + d];
            double ra = s->rho[(size_t)a * M + r], rb = s->rho[(size_t)b * M + r];
            Fa[r] += ra * (ra * fr);
            Fb[r] += rb * (-rb * fr);
          }
        }
        continue;
      }
      const double rr = ramp_ratio(s, i, step);
      for (int side = 0; side < 2; side++) {
        const int src = side == 0 ? b : a, dst = side == 0 ? a : b;
        const cpx* rk = s->rhok + (size_t)src * M;
        for (int d = 0; d < D; d++) {
          /* d_prepareForceKSpace: f_k[dir] * rho_k / M with f_k = -i k u_k */
#pragma omp parallel for schedule(static)
          for (long k = 0; k < M; k++) {
            cpx fk = {0.0, -s->kvec[(size_t)k * D + d] * s->uk[i][k] * rr};
            cpx v = cmul(fk, rk[k]);
            tmp[k].re = v.re / (double)M; tmp[k].im = v.im / (double)M;
          }
          fftnd_exec(&s->F, tmp, +1);
          double* Fd = s->gridF + ((size_t)d * T + dst) * M;
          const double* rd = s->rho + (size_t)dst * M;
#pragma omp parallel for schedule(static)
          for (long r = 0; r < M; r++) Fd[r] += rd[r] * tmp[r].re;
        }
      }
    }
  }
  /* Charges::CalcCharges, pair_style_charges.cu:21-111 */
  if (s->C) {
    const cpx* rk = s->rhok + (size_t)T * M;
    const double a2 = (double)s->cfg.smearing * (double)s->cfg.smearing;
    cpx* psik = s->work2;
    for (long k = 0; k < M; k++) {
      double k2 = s->k2[k];
      if (k2 != 0.0) {
        double g = 4.0 * M_PI * (double)s->cfg.bjerrum / k2 * exp(-k2 / (2.0 * a2)) / (double)M;
        psik[k].re = rk[k].re * g; psik[k].im = rk[k].im * g;
      } else { psik[k].re = 0.0; psik[k].im = 0.0; }
    }
    for (int d = 0; d < D; d++) {
      for (long k = 0; k < M; k++) {
        double kd = s->kvec[(size_t)k * D + d], e = exp(-s->k2[k] / (2.0 * a2));
        tmp[k].re = kd * psik[k].im * e;
        tmp[k].im = -kd * psik[k].re * e;
      }
      fftnd_exec(&s->F, tmp, +1);
      for (long r = 0; r < M; r++) s->Efield[(size_t)d * M + r] = tmp[r].re;
    }
    memcpy(tmp, psik, sizeof(cpx) * (size_t)M);
    fftnd_exec(&s->F, tmp, +1);
    for (long r = 0; r < M; r++) s->psi[r] = tmp[r].re;
  }
  /* gather (device_grid_utils.cu:399-452) + d_bonds (device_bonds.cu:4-60) */
  if (fout) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ns; i++) {
      int li[128]; double lw[128];
      bead_stencil(s, x + i * D, li, lw);
      double f[3] = {0, 0, 0};
      const int t = s->tp[i];
      if (s->C) {
        for (int m = 0; m < S; m++)
          for (int d = 0; d < D; d++) f[d] += s->Efield[(size_t)d * M + li[m]] * lw[m] * s->gvol * (double)s->q[i];
      }
      for (int m = 0; m < S; m++) {
        double r = s->rho[(size_t)t * M + li[m]];
        if (r > 0.0)
          for (int d = 0; d < D; d++) f[d] += s->gridF[((size_t)d * T + t) * M + li[m]] * lw[m] * s->gvol / r;
      }
      for (int bnd = 0; bnd < s->nb[i]; bnd++) {
        int j = s->bto[i * 3 + bnd], bt = s->bty[i * 3 + bnd];
        double dr[3], mdr2 = 0.0;
        for (int d = 0; d < D; d++) {
          float drf = x[i * D + d] - x[(long)j * D + d];
          double v = (double)x[i * D + d] - (double)x[(long)j * D + d];
          if (drf > s->Lh[d]) v -= (double)s->L[d]; else if (drf < -s->Lh[d]) v += (double)s->L[d];
          dr[d] = v; mdr2 += v * v;
        }
        double mf = 0.0;
        if (mdr2 > 1.0e-4) { double mdr = sqrt(mdr2);
          mf = 2.0 * (double)s->cfg.bond_k[bt] * (mdr - (double)s->cfg.bond_req[bt]) / mdr; }
        for (int d = 0; d < D; d++) f[d] -= mf * dr[d];
      }
      for (int d = 0; d < D; d++) fout[i * D + d] = f[d];
    }
  }
  if (rho_out) memcpy(rho_out, s->rho, sizeof(double) * (size_t)(T + s->C) * M);
  s->have_forces = 1;
  s->forces_step = step;
  return TILD_OK;
}

/* Grid force field of the last evaluation divided back by rho where rho > 0, i.e. the
 * quantity the reference gather reads: gridF[d][t][r] / rho_t[r].  out: [T][D][M]. */
int orc_grid_field(orc_sys* s, double* out) {
  const long M = s->M;
  for (int t = 0; t < s->T; t++)
    for (int d = 0; d < s->D; d++)
      for (long r = 0; r < M; r++) {
        double rh = s->rho[(size_t)t * M + r];
        out[((size_t)t * s->D + d) * M + r] = rh > 0.0 ? s->gridF[((size_t)d * s->T + t) * M + r] / rh : 0.0;
      }
  return TILD_OK;
}

/* ---- one step: forces() then Integrate_2() for every integrator (main.cu:298-311) -------- */
int orc_step(orc_sys* s, float* x, float* xo, float* noise, int64_t step, int noise_on, double* fout) {
  const int D = s->D;
  const long ns = s->ns;
  double* f = fout ? fout : (double*)malloc(sizeof(double) * (size_t)ns * D);
  int st = orc_forces(s, x, step, f, NULL);
  if (st) { if (!fout) free(f); return st; }
  const double delt = s->cfg.delt, nmag = s->cfg.noise_mag;
  for (int ig = 0; ig < s->cfg.n_integrators; ig++) {
    const tild_integrator* it = &s->cfg.integrators[ig];
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ns; i++) {
      const int t = s->tp[i];
      if (it->group_type >= 0 && t != it->group_type) continue;
      double z[3] = {0, 0, 0};
      if (noise_on) noise3(s->cfg.seed, (uint32_t)i, step, (uint32_t)ig, z);
      if (it->kind == TILD_INTEGRATOR_GJF) {
        /* d_GJF_integrator, device_GJF_integrator.cu:4-62 */
        const double m = s->cfg.mass[t], Df = s->cfg.diff[t];
        const double b = m / (m + delt / (2.0 * Df));
        const double a = (1.0 - delt / (2.0 * Df * m)) / (1.0 + delt / (2.0 * Df * m));
        for (int j = 0; j < D; j++) {
          const long ai = i * D + j;
          double nn = nmag / Df * z[j];
          float xof = xo[ai];
          if (xof - x[ai] > s->L[j] / 2.0f) xof -= s->L[j];
          else if (xof - x[ai] < -s->L[j] / 2.0f) xof += s->L[j];
          double xn = 2.0 * b * x[ai] - a * xof + b * delt * delt / m * f[ai] + b * delt / (2.0 * m) * (nn + noise[ai]);
          xo[ai] = x[ai];
          noise[ai] = (float)nn;
          float xf = (float)xn;
          if (xf > s->L[j]) xf -= s->L[j]; else if (xf < 0.0f) xf += s->L[j];
          x[ai] = xf;
        }
      } else {
        /* d_EM_integrator, device_EM_integrator.cu:5-36 */
        for (int j = 0; j < D; j++) {
          const long ai = i * D + j;
          float xf = (float)((double)x[ai] + delt * f[ai] + nmag * z[j]);
          if (xf > s->L[j]) xf -= s->L[j]; else if (xf < 0.0f) xf += s->L[j];
          x[ai] = xf;
        }
      }
    }
  }
  if (!fout) free(f);
  return TILD_OK;
}

/* ---- calc_properties(): calc_properties.cu:20-116 ------------------------------------- */
int orc_observables(orc_sys* s, const float* x, tild_obs* o) {
  if (!s->have_forces) return TILD_ERR_STATE;
  const int D = s->D, T = s->T, nP = s->nP;
  const long M = s->M, ns = s->ns;
  memset(o, 0, sizeof(*o));
  o->n_styles = s->cfg.n_styles; o->n_p_comps = nP; o->step = s->forces_step;
  cpx* tmp = s->work;
  double upe = 0.0;
  for (int i = 0; i < s->cfg.n_styles; i++) {
    const tild_pair_style* ps = &s->cfg.styles[i];
    if (ps->style == TILD_STYLE_FIELDPHASE) continue; /* never computed by the reference */
    const int a = ps->type1, b = ps->type2;
    const double rr = ramp_ratio(s, i, s->forces_step);
    const cpx* rkb = s->rhok + (size_t)b * M;
    const double* ra = s->rho + (size_t)a * M;
    /* CalcEnergy: IFFT(u_k rho_b / M), times rho_a, summed, times dV (integ_utils.cu:3-13) */
    for (long k = 0; k < M; k++) { double u = s->uk[i][k] * rr / (double)M; tmp[k].re = u * rkb[k].re; tmp[k].im = u * rkb[k].im; }
    fftnd_exec(&s->F, tmp, +1);
    double e = 0.0;
    for (long r = 0; r < M; r++) e += tmp[r].re * ra[r];
    e *= s->dV;
    o->style_energy[i] = e;
    upe += e;
    /* CalcVirial: IFFT(vir_k * rho_b / M) times rho_a, summed, dV / V / Dim */
    for (int j = 0; j < nP; j++) {
      const cpx* vk = s->virk[i] + (size_t)j * M;
      for (long k = 0; k < M; k++) { cpx r = {rkb[k].re / (double)M, rkb[k].im / (double)M}; tmp[k] = cmul(vk[k], r); }
      fftnd_exec(&s->F, tmp, +1);
      double v = 0.0;
      for (long r = 0; r < M; r++) v += tmp[r].re * ra[r];
      v = v * s->dV / s->V / (double)D;
      o->style_virial[i][j] = v;
      o->ptens[j] += v;
    }
  }
  if (s->C) {
    double e = 0.0;
    for (long r = 0; r < M; r++) e += s->psi[r] * s->rho[(size_t)T * M + r];
    o->uelec = e;
    upe += e;
  }
  /* host_bonds, bonds.cu:3-52 */
  double ub = 0.0, bv[6] = {0, 0, 0, 0, 0, 0};
  for (long i = 0; i < ns; i++) {
    for (int bnd = 0; bnd < s->nb[i]; bnd++) {
      long j = s->bto[i * 3 + bnd];
      if (j < i) continue;
      int bt = s->bty[i * 3 + bnd];
      double dr[3] = {0, 0, 0}, mdr2 = 0.0;
      for (int d = 0; d < D; d++) {
        float drf = x[i * D + d] - x[j * D + d];
        double v = (double)x[i * D + d] - (double)x[j * D + d];
        if (drf > s->Lh[d]) v -= (double)s->L[d]; else if (drf < -s->Lh[d]) v += (double)s->L[d];
        dr[d] = v; mdr2 += v * v;
      }
      double mdr = sqrt(mdr2), delr = mdr - (double)s->cfg.bond_req[bt];
      ub += delr * delr * (double)s->cfg.bond_k[bt];
      double mf = 2.0 * (double)s->cfg.bond_k[bt] * delr / mdr;
      bv[0] += -mf * dr[0] * dr[0];
      bv[1] += -mf * dr[1] * dr[1];
      if (D == 2) bv[2] += -mf * dr[0] * dr[1];
      else { bv[2] += -mf * dr[2] * dr[2]; bv[3] += -mf * dr[0] * dr[1];
             bv[4] += -mf * dr[0] * dr[2]; bv[5] += -mf * dr[1] * dr[2]; }
    }
  }
  for (int j = 0; j < nP; j++) { bv[j] *= 1.0 / s->V / (double)D; o->bond_vir[j] = bv[j]; o->ptens[j] += bv[j]; }
  o->ubond = ub;
  upe += ub;
  o->upe = upe;
  return TILD_OK;
}

/* ---- Compute avg_sk, one call: Compute.cu:83-117 (rho_k * rho_k / M, full spectrum) ---- */
int orc_sk(orc_sys* s, int type, double* out) {
  if (!s->have_forces || type < 0 || type >= s->T) return TILD_ERR_STATE;
  const long M = s->M;
  const cpx* rk = s->rhok + (size_t)type * M;
  for (long k = 0; k < M; k++) { cpx v = cmul(rk[k], rk[k]); out[2 * k] = v.re / (double)M; out[2 * k + 1] = v.im / (double)M; }
  return TILD_OK;
}

/* ---- neighbour list: NList::Initialize / d_assign_cells / d_make_nlist (nlist.cu) ------ */
int orc_nlist(orc_sys* s, const float* x, float rc, int group_type, int32_t* cell_of,
              int32_t* neigh_count, int32_t* neigh, int32_t* cell_max_out) {
  const int D = s->D;
  const long ns = s->ns;
  int nc[3] = {1, 1, 1};
  float Lc[3] = {1, 1, 1};
  int total = 1;
  float cell_vol = 1.0f, V = 1.0f;
  for (int j = 0; j < D; j++) {
    nc[j] = (int)(s->L[j] / rc);
    if (nc[j] < 1) return TILD_ERR_BAD_INPUT;
    Lc[j] = s->L[j] / (int)nc[j];
    total *= nc[j]; cell_vol *= Lc[j]; V *= s->L[j];
  }
  const int cmax = (int)((float)(s->ns * cell_vol / V) * 7.5);
  if (cell_max_out) *cell_max_out = cmax;
  if (!neigh && !neigh_count && !cell_of) return TILD_OK;
  int32_t* cnt = (int32_t*)calloc((size_t)total, 4);
  int32_t* cell_inds = (int32_t*)malloc((size_t)total * (size_t)(cmax > 0 ? cmax : 1) * 4);
  int32_t* pc = (int32_t*)malloc((size_t)ns * 4);
  int overflow = 0;
  for (long i = 0; i < ns; i++) {
    pc[i] = -1;
    if (group_type >= 0 && s->tp[i] != group_type) continue;
    int cid[3] = {0, 0, 0};
    for (int j = 0; j < D; j++) { cid[j] = (int)(x[i * D + j] / Lc[j]); if (cid[j] >= nc[j]) cid[j] -= nc[j]; if (cid[j] < 0) cid[j] += nc[j]; }
    int cn = (D == 2) ? cid[0] + nc[0] * cid[1] : cid[0] + (cid[1] + cid[2] * nc[1]) * nc[0];
    if (cnt[cn] < cmax) cell_inds[(size_t)cn * cmax + cnt[cn]] = (int32_t)i; else overflow = 1;
    cnt[cn]++;
    pc[i] = cn;
  }
  const float rc2 = rc * rc;
  for (long i = 0; i < ns; i++) {
    if (neigh_count) neigh_count[i] = 0;
    if (cell_of) cell_of[i] = pc[i];
    if (pc[i] < 0) continue;
    int nn[3]; int cn = pc[i];
    if (D == 2) { nn[1] = cn / nc[0]; nn[0] = cn % nc[0]; nn[2] = 1; }
    else { nn[2] = cn / (nc[1] * nc[0]); int r = cn - nn[2] * nc[0] * nc[1]; nn[1] = r / nc[0]; nn[0] = r % nc[0]; }
    int ct = 0;
    for (int ix = nn[0] - 1; ix <= nn[0] + 1; ix++) {
      int nix = ix; if (nix < 0) nix = nc[0] - 1; else if (nix == nc[0]) nix = 0;
      for (int iy = nn[1] - 1; iy <= nn[1] + 1; iy++) {
        int niy = iy; if (niy < 0) niy = nc[1] - 1; else if (niy == nc[1]) niy = 0;
        for (int iz = nn[2] - 1; iz <= nn[2] + 1; iz++) {
          int niz = iz;
          if (D == 2) niz = 0; else { if (niz < 0) niz = nc[2] - 1; else if (niz == nc[2]) niz = 0; }
          int ncn = (D == 2) ? nix + nc[0] * niy : nix + (niy + niz * nc[1]) * nc[0];
          int cc = cnt[ncn] < cmax ? cnt[ncn] : cmax;
          for (int q = 0; q < cc; q++) {
            int nid = cell_inds[(size_t)ncn * cmax + q];
            float mdr2 = 0.0f;
            for (int j = 0; j < D; j++) {
              float dr = x[i * D + j] - x[(long)nid * D + j];
              if (dr < -s->Lh[j]) dr += s->L[j]; else if (dr > s->Lh[j]) dr -= s->L[j];
              mdr2 += dr * dr;
            }
            if (mdr2 < rc2) { if (ct < cmax) { if (neigh) neigh[i * cmax + ct] = nid; } else overflow = 1; ct++; }
          }
          if (D == 2) break;
        }
      }
    }
    if (neigh_count) neigh_count[i] = ct;
  }
  free(cnt); free(cell_inds); free(pc);
  return overflow ? TILD_ERR_BAD_INPUT : TILD_OK;
}
