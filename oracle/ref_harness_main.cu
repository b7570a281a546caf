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
//   -nlist rc group: an NList (nlist.cu:13-112) of that group built on the initial positions:
//   <out>_cell.bin d_particle_cell int [ns]; <out>_ncount.bin d_neigh_count int [ns];
//   <out>_neigh.bin d_neigh_inds int [ns][CELL_MAX]; <out>_nlist.txt CELL_MAX total_ncells
//   (the caller checks on the host first that no cell or row overflows CELL_MAX: the reference
//   kernels do not bound their writes)
// Options: -in <script> -out <prefix> [-steps N] [-nonoise] [-ninds K] [-nlist rc group] [-time W]
//   -ninds K dumps the stencils of the first K beads only (large systems)
//   -time W: timing only (no dumps): W untimed steps, then N steps of the reference's main loop
//   with output off (Integrate_1 is a no-op for GJF/EM and check_cudaError only reads the error
//   state, main.cu:104-201), timed with the device synchronised on both sides; prints
//   "harness timing: <N> steps <ms> ms per step"
// Test infrastructure only (it links the reference build); nothing in the product uses it.
#define MAIN
#include "globals.h"
#include "timing.h"
#include <chrono>
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
  std::string nl_group;
  float nl_rc = 0.0f;
  int nsteps = 0, nonoise = 0;
  long long ninds = -1;
  int time_warm = -1;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "-in" && i + 1 < argc) input_file = argv[++i];
    else if (a == "-out" && i + 1 < argc) out = argv[++i];
    else if (a == "-steps" && i + 1 < argc) nsteps = atoi(argv[++i]);
    else if (a == "-nonoise") nonoise = 1;
    else if (a == "-ninds" && i + 1 < argc) ninds = atoll(argv[++i]);
    else if (a == "-time" && i + 1 < argc) time_warm = atoi(argv[++i]);
    else if (a == "-nlist" && i + 2 < argc) {
      nl_rc = (float)atof(argv[++i]);
      nl_group = argv[++i];
    }
  }
  initialize();
  if (nonoise) noise_mag = 0.0f;
  step = 0;
  if (time_warm >= 0) {
    for (step = 1; step <= time_warm; step++) {
      forces();
      for (int i = 0; i < n_integrators; i++) Integrators[i].Integrate_2();
      update_pairstyles();
    }
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < nsteps; k++, step++) {
      forces();
      for (int i = 0; i < n_integrators; i++) Integrators[i].Integrate_2();
      update_pairstyles();
    }
    cudaDeviceSynchronize();
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      fprintf(stderr, "harness: CUDA error %s\n", cudaGetErrorString(e));
      return 1;
    }
    printf("harness timing: %d steps %.6f ms per step\n", nsteps, nsteps > 0 ? ms / nsteps : 0.0);
    return 0;
  }
  dump(out + "_x0.bin", d_x, sizeof(float) * ns * Dim);
  if (!nl_group.empty()) {
    NList nl;
    nl.Initialize(nl_rc, nl_group);
    nl.BuildNList();
    cudaDeviceSynchronize();
    dump(out + "_cell.bin", nl.d_particle_cell, sizeof(int) * ns);
    dump(out + "_ncount.bin", nl.d_neigh_count, sizeof(int) * ns);
    dump(out + "_neigh.bin", nl.d_neigh_inds, sizeof(int) * (size_t)ns * nl.CELL_MAX);
    FILE* f = fopen((out + "_nlist.txt").c_str(), "w");
    fprintf(f, "%d %d\n", nl.CELL_MAX, nl.total_ncells);
    fclose(f);
  }
  forces();
  cudaDeviceSynchronize();
  dump(out + "_f0.bin", d_f, sizeof(float) * ns * Dim);
  dump(out + "_rho0.bin", d_all_rho, sizeof(float) * (size_t)ntypes * M);
  const size_t nst = (ninds >= 0 && ninds < ns) ? (size_t)ninds : (size_t)ns;
  dump(out + "_inds.bin", d_grid_inds, sizeof(int) * nst * grid_per_partic);
  dump(out + "_w.bin", d_grid_W, sizeof(float) * nst * grid_per_partic);
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
