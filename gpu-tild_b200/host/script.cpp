// script.cpp — input script, data file and resume readers (see script.hpp).
#include "script.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

namespace tildhost {

namespace {

[[noreturn]] void die(const std::string& msg) { throw ScriptError(msg); }

// read one pair-style block line: "<keyword> t1 t2 A [Rp] sigma [ramp final]" (read_input.cu:176-416)
StyleLine read_style_line(const std::string& line, const char* keyword, int kind, int ntypes, bool has_rp,
                          bool fieldphase, const char* what) {
  std::istringstream iss2(line);
  std::string convert;
  iss2 >> convert;
  if (convert != keyword) {
    std::cout << "Read: " << convert << " but expected '" << keyword << "' " << std::endl;
    die(std::string("Error in ") + keyword + " section of input file");
  }
  StyleLine st;
  st.kind = kind;
  iss2 >> convert;
  st.type1 = std::stoi(convert) - 1;
  iss2 >> convert;
  st.type2 = std::stoi(convert) - 1;
  iss2 >> convert;
  st.initial_prefactor = std::stof(convert);
  st.final_prefactor = st.initial_prefactor;
  if (fieldphase) {
    iss2 >> convert;
    st.phase = std::stoi(convert);
    iss2 >> convert;
    st.dir = std::stoi(convert);
    iss2 >> convert;
    st.n_periods = std::stoi(convert);
  } else {
    if (has_rp) {
      iss2 >> convert;
      st.rp = std::stof(convert);
    }
    iss2 >> convert;
    st.sigma_squared = std::stof(convert);
    st.sigma_squared *= st.sigma_squared;
  }
  if (st.type1 >= ntypes || st.type2 >= ntypes) die(std::string("Invalid particle type in ") + what + " input!");
  if (iss2.tellg() != -1) {
    iss2 >> convert;
    if (convert == "ramp") {
      st.ramp = true;
      iss2 >> convert;
      st.final_prefactor = std::stof(convert);
    }
  }
  return st;
}

void skip_line(FILE* f) {
  char tt[120];
  if (!fgets(tt, 120, f)) tt[0] = 0;
}

}  // namespace

// ---- read_config / read_charge_config (config_utils.cu:5-364) ----------------------------------
void read_config(const std::string& path, Script& s, bool with_charges) {
  FILE* inp = fopen(path.c_str(), "r");
  if (!inp) die("Failed to open " + path + "!");
  System& y = s.sys;
  const int Dim = s.Dim;
  skip_line(inp);
  skip_line(inp);
  int ok = 1;
  ok &= fscanf(inp, "%d", &y.ns) == 1; skip_line(inp);
  ok &= fscanf(inp, "%d", &y.n_total_bonds) == 1; skip_line(inp);
  ok &= fscanf(inp, "%d", &y.n_total_angles) == 1; skip_line(inp);
  skip_line(inp);
  ok &= fscanf(inp, "%d", &y.ntypes) == 1; skip_line(inp);
  ok &= fscanf(inp, "%d", &y.nbond_types) == 1; skip_line(inp);
  ok &= fscanf(inp, "%d", &y.nangle_types) == 1; skip_line(inp);
  skip_line(inp);
  for (int d = 0; d < 3; d++) {
    if (with_charges) {
      float lo = 0, hi = 0;
      ok &= fscanf(inp, "%f %f", &lo, &hi) == 2;
      y.L[d] = (float)(hi - lo);
    } else {
      double lo = 0, hi = 0;
      ok &= fscanf(inp, "%lf %lf", &lo, &hi) == 2;
      y.L[d] = (float)(hi - lo);
    }
    skip_line(inp);
  }
  if (!ok || y.ns <= 0 || y.ntypes <= 0) {
    fclose(inp);
    die("Malformed header in " + path);
  }
  if (Dim <= 2) y.L[2] = 1.0f;
  y.mass.assign(y.ntypes, 0.f);
  y.diff.assign(y.ntypes, 1.0f);
  y.tp.assign(y.ns, 0);
  y.molecID.assign(y.ns, 0);
  y.x.assign((size_t)y.ns * Dim, 0.f);
  y.n_bonds.assign(y.ns, 0);
  y.bonded_to.assign((size_t)y.ns * 3, 0);
  y.bond_type.assign((size_t)y.ns * 3, 0);
  y.bond_k.assign(std::max(y.nbond_types, 0), 0.f);
  y.bond_req.assign(std::max(y.nbond_types, 0), 0.f);
  if (with_charges) y.charges.assign(y.ns, 0.f);
  skip_line(inp);
  skip_line(inp);
  skip_line(inp);
  for (int i = 0; i < y.ntypes; i++) {
    int di = 0;
    if (with_charges) {
      float m = 0;
      if (fscanf(inp, "%d %f", &di, &m) != 2) die("Malformed Masses section");
      if (di >= 1 && di <= y.ntypes) y.mass[di - 1] = m;
    } else {
      double m = 0;
      if (fscanf(inp, "%d %lf", &di, &m) != 2) die("Malformed Masses section");
      if (di >= 1 && di <= y.ntypes) y.mass[di - 1] = (float)m;
    }
    skip_line(inp);
  }
  skip_line(inp);
  skip_line(inp);
  skip_line(inp);
  for (int i = 0; i < y.ns; i++) {
    if (feof(inp)) die("Premature end of input.conf!");
    int ind = 0, di = 0, ltp = 0;
    if (fscanf(inp, "%d %d %d", &ind, &di, &ltp) != 3) die("Premature end of input.conf!");
    ind -= 1;
    if (ind < 0 || ind >= y.ns) die("atom id out of range in " + path);
    if (ltp < 1 || ltp > y.ntypes) die("atom type out of range in " + path);
    y.molecID[ind] = di - 1;
    y.tp[ind] = ltp - 1;
    if (with_charges) {
      float q = 0;
      if (fscanf(inp, "%f", &q) != 1) die("Premature end of input.conf!");
      y.charges[ind] = q;
      for (int j = 0; j < Dim; j++) {
        float v = 0;
        if (fscanf(inp, "%f", &v) != 1) die("Premature end of input.conf!");
        y.x[(size_t)ind * Dim + j] = v;
      }
    } else {
      for (int j = 0; j < Dim; j++) {
        double v = 0;
        if (fscanf(inp, "%lf", &v) != 1) die("Premature end of input.conf!");
        y.x[(size_t)ind * Dim + j] = (float)v;
      }
    }
    skip_line(inp);
  }
  skip_line(inp);
  skip_line(inp);
  skip_line(inp);
  for (int i = 0; i < y.n_total_bonds; i++) {
    if (feof(inp)) die("Premature end of input.conf!");
    int di = 0, bt = 0, a = 0, b = 0;
    if (fscanf(inp, "%d", &di) != 1 || fscanf(inp, "%d", &bt) != 1 || fscanf(inp, "%d", &a) != 1 ||
        fscanf(inp, "%d", &b) != 1)
      die("Premature end of input.conf!");
    int i1 = a - 1, i2 = b - 1, btype = bt - 1;
    if (i2 < i1) std::swap(i1, i2);
    if (i1 < 0 || i2 >= y.ns) die("bond atom out of range in " + path);
    if (y.n_bonds[i1] >= TILD_MAX_BONDS || y.n_bonds[i2] >= TILD_MAX_BONDS)
      die("more than MAX_BONDS (3) bonds on one atom");
    y.bonded_to[(size_t)i1 * 3 + y.n_bonds[i1]] = i2;
    y.bond_type[(size_t)i1 * 3 + y.n_bonds[i1]] = btype;
    y.n_bonds[i1]++;
    y.bonded_to[(size_t)i2 * 3 + y.n_bonds[i2]] = i1;
    y.bond_type[(size_t)i2 * 3 + y.n_bonds[i2]] = btype;
    y.n_bonds[i2]++;
  }
  fclose(inp);
}

// ---- read_resume (config_utils.cu:405-454): positions by line order --------------------------
// The header is skipped as the reference skips it.  Atom lines ("id type mol x y z [q]", the
// trajectory format of write_lammps_traj, config_utils.cu:366-403) are read one line at a time:
// the reference's "%f " after the last coordinate also consumes the newline, so in 3-D frames
// without charges its fgets(tt, 5) then eats the start of the next line; reading whole lines
// takes every frame the reference writes, 2-D, 3-D, with and without charges.
void read_resume(const std::string& path, Script& s) {
  FILE* inp = fopen(path.c_str(), "r");
  if (!inp) die("Failed to open " + path + "!");
  char tt[120];
  for (int k = 0; k < 3; k++)
    if (!fgets(tt, 100, inp)) break;
  int ns_tmp = -1;
  if (fscanf(inp, "%d", &ns_tmp) != 1 || ns_tmp != s.sys.ns) {
    fclose(inp);
    die("number of sites in resume file doesn't match input!");
  }
  for (int k = 0; k < 6; k++)
    if (!fgets(tt, 100, inp)) break;
  const int Dim = s.Dim;
  char line[512];
  for (int i = 0; i < s.sys.ns; i++) {
    if (!fgets(line, sizeof line, inp)) {
      fclose(inp);
      die("Premature end of resume file");
    }
    int t1, t2, t3, used = 0;
    const char* q = line;
    if (sscanf(q, "%d %d %d%n", &t1, &t2, &t3, &used) != 3) {
      fclose(inp);
      die("Premature end of resume file");
    }
    q += used;
    for (int j = 0; j < Dim; j++) {
      if (sscanf(q, "%f%n", &s.sys.x[(size_t)i * Dim + j], &used) != 1) {
        fclose(inp);
        die("Premature end of resume file");
      }
      q += used;
    }
  }
  fclose(inp);
  std::cout << "SUCCESSFULLY READ RESUME FILE" << std::endl;
}

// ---- read_input (read_input.cu:12-533) ---------------------------------------------------------
Script parse_script(const std::string& path, int seed_default) {
  Script s;
  // set_defaults (read_input.cu:536-562)
  s.Dim = 2;
  s.delt = 0.005f;
  s.pmeorder = 1;
  s.Nx[0] = s.Nx[1] = 35;
  s.threads = 512;
  s.noise_mag = sqrtf(2.0f * s.delt);
  s.max_steps = 100000;
  s.rand_seed = seed_default;
  s.log_freq = 2500;
  s.grid_freq = 0;
  s.traj_freq = 0;
  s.struc_freq = 0;
  s.skip_steps = 20000;
  s.bin_freq = 5000;
  s.dump_name = "traj.lammpstrj";

  std::ifstream in2(path);
  if (!in2) die("Failed to open input script " + path);
  std::string word, line;
  bool config_read = false, read_charge_flag = false;
  while (std::getline(in2, line)) {
    if (line.length() == 0 || line.at(0) == '#') continue;
    std::istringstream iss(line);
    while (iss >> word) {
      if (word == "binary_freq") {
        std::string v; iss >> v; s.bin_freq = std::stoi(v);
      } else if (word == "bond") {
        if (!config_read) die("Error in input file, bond keyword before config read");
        std::string a, test, k, r;
        iss >> a;
        const int btype = std::stoi(a);
        iss >> test;
        if (test != "harmonic") die("You fool! That bond type is not supported!");
        iss >> k >> r;
        if (btype < 1 || btype > (int)s.sys.bond_k.size()) die("bond type out of range");
        s.sys.bond_k[btype - 1] = std::stof(k);
        s.sys.bond_req[btype - 1] = std::stof(r);
      } else if (word == "charges") {
        if (config_read) die("charges keyword must come before read_data command!");
        read_charge_flag = true;
        std::string a, b;
        iss >> a >> b;
        s.bjerrum = std::stof(a);
        s.smearing = std::stof(b);
        s.do_charges = true;
      } else if (word == "compute") {
        ComputeDef c;
        c.input_command = line;
        std::istringstream ic(line);
        std::string w;
        ic >> w >> w;
        if (w != "avg_sk") die("Undefined compute style!");
        c.style = w;
        ic >> w;
        c.type = std::stoi(w) - 1;
        if (c.type >= s.sys.ntypes) die("Invalid type to calculate avg_sk");
        while (ic >> w) {
          if (w == "freq") { ic >> w; c.freq = std::stoi(w); }
          else if (w == "wait") { ic >> w; c.wait = std::stoi(w); }
        }
        std::cout << "  Calculating <S(k)> for component " << c.type + 1 << " every " << c.freq << " steps after "
                  << c.wait << " steps have passed." << std::endl;
        s.computes.push_back(c);
        while (iss >> word) {}
      } else if (word == "delt") {
        std::string v; iss >> v;
        s.delt = std::stof(v);
        s.noise_mag = sqrtf(2.f * s.delt);
      } else if (word == "diffusivity") {
        if (!config_read) die("Error in input file, diffusivities defined before config read");
        std::string a, b;
        iss >> a >> b;
        const int atype = std::stoi(a);
        if (atype > s.sys.ntypes || atype < 1) die("Invalid type for diffusivity!");
        s.sys.diff[atype - 1] = std::stof(b);
      } else if (word == "Dim") {
        std::string v; iss >> v; s.Dim = std::stoi(v);
      } else if (word == "grid_freq") {
        std::string v; iss >> v; s.grid_freq = std::stoi(v);
      } else if (word == "group") {
        if (!config_read) die("Must read the configuration file before defining a group!");
        GroupDef g;
        iss >> word;
        g.name = word;
        iss >> word;
        g.command_line = line;
        if (word == "type") {
          std::string v; iss >> v;
          g.type = std::stoi(v) - 1;
        } else {
          die("ERROR: Group type " + word + " not supported!");
        }
        s.groups.push_back(g);
      } else if (word == "integrator") {
        if (!config_read) die("Integrator must be defined after read_data command!");
        IntegratorDef it;
        iss >> it.group >> it.name;
        if (it.name != "EM" && it.name != "GJF") die(it.name + " is not a valid integrator!");
        it.group_index = -1;
        for (size_t i = 0; i < s.groups.size(); i++)
          if (s.groups[i].name == it.group) it.group_index = (int)i;
        if (it.group_index == -1) die("Group " + it.group + " not found to integrate!");
        if (it.name == "GJF") s.using_gjf = true;
        s.integrators.push_back(it);
      } else if (word == "log_freq") {
        std::string v; iss >> v; s.log_freq = std::stoi(v);
      } else if (word == "max_steps") {
        std::string v; iss >> v; s.max_steps = std::stoi(v);
      } else if (word == "n_erfs" || word == "n_gaussians" || word == "n_gaussian_erfs" || word == "n_fieldphases") {
        std::string v; iss >> v;
        const int n = std::stoi(v);
        std::vector<StyleLine>* dst;
        const char* kw;
        int kind;
        bool rp = false, fp = false;
        const char* what;
        if (word == "n_erfs") { dst = &s.erfs; kw = "erf"; kind = TILD_STYLE_ERF; rp = true; what = "Erf potential"; }
        else if (word == "n_gaussians") { dst = &s.gaussians; kw = "gaussian"; kind = TILD_STYLE_GAUSSIAN; what = "Gaussian"; }
        else if (word == "n_gaussian_erfs") { dst = &s.gauss_erfs; kw = "gaussian_erf"; kind = TILD_STYLE_GAUSSIAN_ERF; rp = true; what = "GaussianErf potential"; }
        else { dst = &s.fieldphases; kw = "fieldphase"; kind = TILD_STYLE_FIELDPHASE; fp = true; what = "FieldPhase potential"; }
        dst->clear();
        for (int i = 0; i < n; i++) {
          if (!std::getline(in2, line)) die(std::string("Error in ") + kw + " section of input file");
          dst->push_back(read_style_line(line, kw, kind, s.sys.ntypes, rp, fp, what));
        }
      } else if (word == "Nx") {
        std::string v; iss >> v; s.Nx[0] = std::stoi(v);
      } else if (word == "Ny") {
        std::string v; iss >> v; s.Nx[1] = std::stoi(v);
      } else if (word == "Nz") {
        std::string v; iss >> v;
        if (s.Dim > 2) s.Nx[2] = std::stoi(v);
      } else if (word == "pmeorder") {
        std::string v; iss >> v;
        s.pmeorder = std::stoi(v);
        if (s.pmeorder > 4) die("PMEORDER greater than 4 not supported!");
      } else if (word == "rand_seed") {
        std::string v; iss >> v; s.rand_seed = std::stoi(v);
      } else if (word == "read_data") {
        std::string v; iss >> v;
        if (read_charge_flag) std::cout << "READING CHARGE CONFIG" << std::endl;
        read_config(v, s, read_charge_flag);
        config_read = true;
        s.groups.clear();
        GroupDef all;
        all.name = "all";
        all.command_line = "NONE";
        s.groups.push_back(all);
      } else if (word == "read_resume") {
        std::string v; iss >> v;
        read_resume(v, s);
        s.read_resume = true;
        s.resume_name = v;
      } else if (word == "skip_steps") {
        std::string v; iss >> v; s.skip_steps = std::stoi(v);
      } else if (word == "struc_freq") {
        std::string v; iss >> v; s.struc_freq = std::stoi(v);
      } else if (word == "threads") {
        std::string v; iss >> v; s.threads = std::stoi(v);
      } else if (word == "traj_freq") {
        std::string v; iss >> v; s.traj_freq = std::stoi(v);
      } else if (word == "traj_name") {
        s.dump_name.clear();
        iss >> s.dump_name;
      } else {
        std::cout << "Invalid keyword: " << word << std::endl;
        die("Invalid keyword error");
      }
    }
    s.echoed.push_back(line);
    std::cout << line << std::endl;
  }
  if (!config_read) die("no read_data command in the input script");
  if (s.using_gjf && s.delt < 0.002f) {
    std::cout << "WARNING!!!!! WARNING!!!! WARNING!!!!" << std::endl;
    std::cout << "Previous tests have seen problems with GJF algorithm and time steps < 0.002" << std::endl;
  }
  return s;
}

// ---- write_runtime_parameters (read_input.cu:565-651) -------------------------------------------
std::string runtime_parameters(const Script& s) {
  std::ostringstream otp;
  otp << "Dim " << s.Dim << std::endl;
  otp << "Nx " << s.Nx[0] << std::endl;
  otp << "Ny " << s.Nx[1] << std::endl;
  if (s.Dim == 3) otp << "Nz " << s.Nx[2] << std::endl;
  otp << "delt " << s.delt << std::endl;
  for (size_t i = 1; i < s.groups.size(); i++) otp << s.groups[i].command_line << std::endl;
  for (const auto& it : s.integrators) otp << "integrator " << s.groups.at(it.group_index).name << " " << it.name << std::endl;
  otp << "rand_seed " << s.rand_seed << std::endl;
  if (s.read_resume) otp << "read_resume " << s.resume_name << std::endl;
  otp << "max_steps " << s.max_steps << std::endl;
  otp << "log_freq " << s.log_freq << std::endl;
  otp << "threads " << s.threads << std::endl;
  otp << "grid_freq " << s.grid_freq << std::endl;
  otp << "traj_freq " << s.traj_freq << std::endl;
  otp << "binary_freq " << s.bin_freq << std::endl;
  otp << "struc_freq " << s.struc_freq << std::endl;
  otp << "skip_steps " << s.skip_steps << std::endl;
  otp << "pmeorder " << s.pmeorder << std::endl;
  if (s.do_charges) otp << "charges " << s.bjerrum << " " << s.smearing << std::endl;
  for (int i = 0; i < s.sys.ntypes; i++) otp << "diffusivity " << i + 1 << " " << s.sys.diff[i] << std::endl;
  if (!s.gaussians.empty()) {
    otp << "n_gaussians " << s.gaussians.size() << std::endl;
    for (const auto& g : s.gaussians)  // the reference prints no space after "gaussian"
      otp << "gaussian" << g.type1 + 1 << " " << g.type2 + 1 << " " << g.initial_prefactor << " " << g.sigma_squared
          << std::endl;
  }
  if (!s.fieldphases.empty()) {
    otp << "n_fieldphases " << s.fieldphases.size() << std::endl;
    for (const auto& f : s.fieldphases)
      otp << "fieldphase " << f.type1 + 1 << " " << f.type2 + 1 << " " << f.initial_prefactor << " " << f.phase << " "
          << f.dir << " " << f.n_periods << std::endl;
  }
  if (!s.erfs.empty()) {
    otp << "n_erfs " << s.erfs.size() << std::endl;
    for (const auto& e : s.erfs)
      otp << "erf " << e.type1 + 1 << " " << e.type2 + 1 << " " << e.initial_prefactor << " " << e.rp << " "
          << e.sigma_squared << std::endl;
    otp << std::endl;
  }
  if (!s.gauss_erfs.empty()) {
    otp << "n_gaussian_erfs " << s.gauss_erfs.size() << std::endl;
    for (const auto& e : s.gauss_erfs)  // printed with the "erf" keyword, as the reference does
      otp << "erf " << e.type1 + 1 << " " << e.type2 + 1 << " " << e.initial_prefactor << " " << e.rp << " "
          << e.sigma_squared << std::endl;
    otp << std::endl;
  }
  for (const auto& c : s.computes) otp << c.input_command << std::endl;
  for (int i = 0; i < s.sys.nbond_types; i++)
    otp << "bond " << i + 1 << " harmonic " << s.sys.bond_k[i] << " " << s.sys.bond_req[i] << std::endl;
  return otp.str();
}

tild_config make_config(const Script& s) {
  tild_config c;
  memset(&c, 0, sizeof(c));
  const System& y = s.sys;
  c.dim = s.Dim;
  for (int d = 0; d < 3; d++) {
    c.nx[d] = d < s.Dim ? s.Nx[d] : 1;
    c.box[d] = d < s.Dim ? y.L[d] : 1.0f;
  }
  c.ns = y.ns;
  c.ntypes = y.ntypes;
  c.pmeorder = s.pmeorder;
  c.delt = s.delt;
  c.noise_mag = s.noise_mag;
  c.seed = (uint64_t)(uint32_t)s.rand_seed;
  c.rng = TILD_RNG_PHILOX;
  c.max_steps = s.max_steps;
  auto add = [&](const StyleLine& l) {
    if (c.n_styles >= TILD_MAX_STYLES) throw ScriptError("too many pair styles");
    tild_pair_style& p = c.styles[c.n_styles++];
    p.style = l.kind;
    p.type1 = l.type1;
    p.type2 = l.type2;
    p.ramp = l.ramp;
    p.prefactor = (float)l.initial_prefactor;
    p.final_prefactor = (float)l.final_prefactor;
    p.sigma = (float)std::sqrt(l.sigma_squared);
    p.rp = (float)l.rp;
    p.phase = l.phase;
    p.dir = l.dir;
    p.n_periods = l.n_periods;
  };
  for (const auto& l : s.gaussians) add(l);
  for (const auto& l : s.erfs) add(l);
  for (const auto& l : s.fieldphases) add(l);
  for (const auto& l : s.gauss_erfs) add(l);
  c.do_charges = s.do_charges;
  c.bjerrum = s.bjerrum;
  c.smearing = s.smearing;
  if (y.nbond_types > TILD_MAX_BOND_TYPES) throw ScriptError("too many bond types");
  c.n_bond_types = y.nbond_types;
  for (int b = 0; b < y.nbond_types; b++) {
    c.bond_k[b] = y.bond_k[b];
    c.bond_req[b] = y.bond_req[b];
  }
  if (y.ntypes > TILD_MAX_TYPES) throw ScriptError("too many particle types");
  for (int t = 0; t < y.ntypes; t++) {
    c.mass[t] = y.mass[t];
    c.diff[t] = y.diff[t];
  }
  if ((int)s.integrators.size() > TILD_MAX_INTEGRATORS) throw ScriptError("too many integrators");
  c.n_integrators = (int)s.integrators.size();
  for (size_t k = 0; k < s.integrators.size(); k++) {
    c.integrators[k].kind = s.integrators[k].name == "GJF" ? TILD_INTEGRATOR_GJF : TILD_INTEGRATOR_EM;
    c.integrators[k].group_type = s.groups.at(s.integrators[k].group_index).type;
  }
  c.table_mode = TILD_TABLES_FP64;
  return c;
}

}  // namespace tildhost
