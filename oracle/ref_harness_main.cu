// ref_harness_main.cu — test harness around the unmodified reference objects (everything
// except its main.o).  The reference writes no forces to any file, so this main runs its own
// initialize() and forces() and dumps the device arrays the parity tests compare:
//   <out>_x0.bin   positions after initialize()            float [ns][Dim]
//   <out>_f0.bin   d_f after forces()                       float [ns][Dim]
//   <out>_rho0.bin d_all_rho after forces()                 float [ntypes][M]
//   <out>_inds.bin d_grid_inds                              int   [ns][grid_per_partic]
//   <out>_w.bin    d_grid_W                                 float [ns][grid_per_partic]
//   <out>_obs0.txt calc_properties(): Upe Ubond Ptens... per-style energies
//   <out>_xN.bin / <out>_fN.bin after N steps of forces(); Integrate_2(); update_pairstyles()
// Options: -in <script> -out <prefix> [-steps N] [-nonoise]
// Test infrastructure only (it links the reference build); nothing in the product uses it.
#define MAIN
#include "globals.h"
#include "timing.h"
#include <cstdio>
#include <string>

void forces(void);
void initialize(void);
void calc_properties(void);
void update_pairstyles(void);
void cuda_collect_x(void);

static void dump(const std::string& name, const void* dev, size_t bytes) {
  std::vector<char> h(bytes);
  cudaMemcpy(h.data(), dev, bytes, cudaMemcpyDeviceToHost);
  FILE* f = fopen(name.c_str(), "wb");
  fwrite(h.data(), 1, bytes, f);
  fclose(f);
}

static void dump_obs(const std::string& name) {
  FILE* f = fopen(name.c_str(), "w");
  fprintf(f, "%.9e %.9e", (double)Upe, (double)Ubond);
  for (int i = 0; i < n_P_comps; i++) fprintf(f, " %.9e", (double)Ptens[i]);
  for (Gaussian& g : Gausses) fprintf(f, " %.9e", (double)g.energy);
  for (Erf& g : Erfs) fprintf(f, " %.9e", (double)g.energy);
  for (GaussianErf& g : GaussErfs) fprintf(f, " %.9e", (double)g.energy);
  if (do_charges) fprintf(f, " %.9e", (double)*electrostatic_energy);
  fprintf(f, "\n");
  fclose(f);
}

int main(int argc, char** argv) {
  std::string out = "ref";
  int nsteps = 0, nonoise = 0;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "-in" && i + 1 < argc) input_file = argv[++i];
    else if (a == "-out" && i + 1 < argc) out = argv[++i];
    else if (a == "-steps" && i + 1 < argc) nsteps = atoi(argv[++i]);
    else if (a == "-nonoise") nonoise = 1;
  }
  initialize();
  if (nonoise) noise_mag = 0.0f;
  step = 0;
  dump(out + "_x0.bin", d_x, sizeof(float) * ns * Dim);
  forces();
  cudaDeviceSynchronize();
  dump(out + "_f0.bin", d_f, sizeof(float) * ns * Dim);
  dump(out + "_rho0.bin", d_all_rho, sizeof(float) * (size_t)ntypes * M);
  dump(out + "_inds.bin", d_grid_inds, sizeof(int) * (size_t)ns * grid_per_partic);
  dump(out + "_w.bin", d_grid_W, sizeof(float) * (size_t)ns * grid_per_partic);
  calc_properties();
  dump_obs(out + "_obs0.txt");
  for (step = 1; step <= nsteps; step++) {
    forces();
    for (int i = 0; i < n_integrators; i++) Integrators[i].Integrate_2();
    update_pairstyles();
  }
  if (nsteps > 0) {
    cudaDeviceSynchronize();
    char nm[64];
    snprintf(nm, sizeof nm, "_x%d.bin", nsteps);
    dump(out + nm, d_x, sizeof(float) * ns * Dim);
    step = nsteps;
    forces();
    cudaDeviceSynchronize();
    snprintf(nm, sizeof nm, "_f%d.bin", nsteps);
    dump(out + nm, d_f, sizeof(float) * ns * Dim);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "harness: CUDA error %s\n", cudaGetErrorString(e));
    return 1;
  }
  printf("harness ok: ns=%d M=%d steps=%d\n", ns, M, nsteps);
  return 0;
}
