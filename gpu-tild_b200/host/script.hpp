// script.hpp — the input-script and data-file surface of gpu-tild, host side.
//
// Parses the keyword grammar of read_input() (read_input.cu:12-533) with its defaults
// (set_defaults, :536-562) and ordering rules, reads the fixed-layout data files
// (read_config / read_charge_config, config_utils.cu:5-364) and resume frames
// (read_resume, :405-454).  Errors are reported the way the reference's die() words them,
// but as exceptions: nothing here exits the process.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>
#include "../../include/tild.h"

namespace tildhost {

struct ScriptError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct StyleLine {                // one pair-style line as read (types 0-based)
  int kind = 0;
  int type1 = 0, type2 = 0;
  double initial_prefactor = 0, final_prefactor = 0;
  double sigma_squared = 0, rp = 0;
  int phase = 0, dir = 0, n_periods = 0;
  bool ramp = false;
};

struct GroupDef {
  std::string name;
  std::string command_line;
  int type = -1;                  // -1: "all"
};

struct IntegratorDef {
  std::string group;
  std::string name;               // "EM" | "GJF"
  int group_index = 0;
};

struct ComputeDef {
  std::string input_command;
  std::string style;              // "avg_sk"
  int type = 0;
  int freq = 100, wait = 0;
};

struct System {
  // topology / configuration (read_config)
  int ns = 0, n_total_bonds = 0, n_total_angles = 0, ntypes = 0, nbond_types = 0, nangle_types = 0;
  float L[3] = {1, 1, 1};
  std::vector<float> mass, diff;
  std::vector<int> tp, molecID;
  std::vector<float> charges;     // empty unless do_charges
  std::vector<float> x;           // [ns * Dim]
  std::vector<int> n_bonds, bonded_to, bond_type;  // [ns], [ns*3], [ns*3]
  std::vector<float> bond_k, bond_req;
};

struct Script {
  // values of the globals after read_input()
  int Dim = 2;
  float delt = 0.005f;
  float noise_mag = 0.f;
  int pmeorder = 1;
  int Nx[3] = {35, 35, 0};
  int threads = 512;
  int max_steps = 100000;
  int rand_seed = 0;
  int log_freq = 2500, grid_freq = 0, traj_freq = 0, struc_freq = 0, skip_steps = 20000, bin_freq = 5000;
  std::string dump_name = "traj.lammpstrj";
  bool do_charges = false;
  float bjerrum = 0.f, smearing = 0.f;
  bool read_resume = false;
  std::string resume_name;
  std::vector<StyleLine> gaussians, erfs, gauss_erfs, fieldphases;
  std::vector<GroupDef> groups;   // groups[0] = "all"
  std::vector<IntegratorDef> integrators;
  std::vector<ComputeDef> computes;
  std::vector<std::string> echoed;  // every line, echoed as read_input prints it
  System sys;
  bool using_gjf = false;
};

// Parses `path` (relative data/resume names resolve against the current directory, as in the
// reference).  seed_default is used when the script has no rand_seed (reference: time(0)).
Script parse_script(const std::string& path, int seed_default);

void read_config(const std::string& path, Script& s, bool with_charges);
void read_resume(const std::string& path, Script& s);

// NEED_A_NAME.input text (write_runtime_parameters, read_input.cu:565-651), quirks included.
std::string runtime_parameters(const Script& s);

// tild_config for the parsed script (styles in the reference's evaluation order).
tild_config make_config(const Script& s);

}  // namespace tildhost
