// solver.h -- the ATUS-2 solver classes on top of libatus_gpu.so.
//
// CRT_Base, CRT_Base_IF and CSOB_Base keep the public interface, the XML
// semantics, the console output and the files of the reference's class
// templates (include/CRT_Base.h, include/CRT_Base_IF.h, include/CRT_Base_IF_2.h,
// include/CSOB_Base.h),
// while the fields live on the GPU: the step functions and the Strang block of
// run_sequence go through the C ABI (include/atus_gpu.h).  A host copy of the
// fields (Getp2In) is refreshed only when a file is written or a host-side step
// function (a user's StepFunction) needs it, and uploaded again afterwards.
//
// GPU step tags: "freeprop" (CRT_Base: V + g|psi|^2; CRT_Base_IF: g|psi|^2 +
// beta.x - DeltaL), CRT_Base_IF's numerical "bragg" and "raman", and those a
// subclass adds to m_gpu_steps (e.g. "bragg_ad").
// Any other tag is looked up in m_map_stepfcts and runs on the host copy.
#pragma once

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <list>
#include <map>
#include <string>
#include <vector>

#include "atus_gpu.h"
#include "expr.h"
#include "my_structs.h"
#include "params.h"

namespace atus {

using fftw_complex = double[2];
template <int dim> using CPoint = std::array<double, dim>;

template <int dim> double dot(const CPoint<dim> &a, const CPoint<dim> &b) {
  double r = 0;
  for (int i = 0; i < dim; i++) r += a[i] * b[i];
  return r;
}

inline void gpu_check(atus_ctx *ctx, int r, const char *what) {
  if (r != ATUS_OK)
    throw std::string(std::string("GPU error in ") + what + ": " + (ctx ? atus_last_error(ctx) : "no context") +
                      " (code " + std::to_string(r) + ")");
}

typedef void (*StepFunction)(void *, sequence_item &);

// Grid geometry of a header (CRT_shared::Read_header, include/CRT_shared.h:131-172).
template <int dim> struct Grid {
  generic_header h{};
  int64_t npts = 0;
  int shift[3] = {0, 0, 0};
  double ar = 0, ar_k = 0;
  void setup() {
    if (dim == 1) { h.nDimY = 1; h.nDimZ = 1; }
    if (dim == 2) h.nDimZ = 1;
    npts = h.nDimX * h.nDimY * h.nDimZ;
    shift[0] = (int)(h.nDimX / 2);
    shift[1] = (int)(h.nDimY / 2);
    shift[2] = (int)(h.nDimZ / 2);
    ar = h.dx;
    ar_k = h.dkx;
    if (dim >= 2) { ar *= h.dy; ar_k *= h.dky; }
    if (dim >= 3) { ar *= h.dz; ar_k *= h.dkz; }
  }
  // x_i = (i - N/2) dx (cft_3d.cpp:128-138)
  CPoint<dim> Get_x(int64_t l) const {
    const int64_t i = l / (h.nDimY * h.nDimZ), j = (l / h.nDimZ) % h.nDimY, k = l % h.nDimZ;
    CPoint<dim> x{};
    const int64_t idx[3] = {i, j, k};
    const double d[3] = {h.dx, h.dy, h.dz};
    for (int a = 0; a < dim; a++) x[a] = double(idx[a] - shift[a]) * d[a];
    return x;
  }
  atus_grid abi() const {
    atus_grid g{};
    g.dim = dim;
    g.n[0] = h.nDimX;
    g.n[1] = dim >= 2 ? h.nDimY : 1;
    g.n[2] = dim >= 3 ? h.nDimZ : 1;
    g.d[0] = h.dx; g.d[1] = h.dy; g.d[2] = h.dz;
    g.dk[0] = h.dkx; g.dk[1] = h.dky; g.dk[2] = h.dkz;
    g.t = h.t;
    return g;
  }
};

// ============================================================== CRT_Base
template <int dim, int no_int_states>
class CRT_Base {
 public:
  explicit CRT_Base(ParameterHandler *params, int precision = ATUS_PREC_FP64) : m_params(params) {
    // Read_header + LoadFiles (include/CRT_Base.h:143-148, 206-240)
    m_grid.h = read_header(params->Get_simulation("FILENAME"));
    if (m_grid.h.nDims != dim) throw std::string("header.nDims does not match the program dimension");
    m_grid.setup();
    for (int c = 0; c < no_int_states; c++) m_fields[c].assign(2 * m_grid.npts, 0.0);
    load(params->Get_simulation("FILENAME"), 0);
    for (int c = 1; c < no_int_states; c++) load(params->Get_simulation("FILENAME_" + std::to_string(c + 1)), c);
    const atus_grid g = m_grid.abi();
    gpu_check(nullptr, atus_create(&g, no_int_states, precision, &m_gpu), "atus_create");
    for (int c = 0; c < no_int_states; c++)
      gpu_check(m_gpu, atus_upload_psi(m_gpu, c, m_fields[c].data()), "upload");
    // Init() runs here, before Alpha_1 is read (include/CRT_Base.h:149, 171-173)
    gpu_check(m_gpu, atus_set_dt(m_gpu, m_grid.h.dt), "set_dt");
    m_gpu_steps["freeprop"] = ATUS_STEP_NL;
    for (int i = 0; i < no_int_states; i++)
      for (int j = 0; j < no_int_states; j++)
        m_gs[j + no_int_states * i] = m_params->Get_VConstant("GS_" + std::to_string(i + 1), j);
    gpu_check(m_gpu, atus_set_gs(m_gpu, m_gs.data()), "set_gs");
    for (int i = 0; i < dim; i++) m_alpha[i] = m_params->Get_VConstant("Alpha_1", i);
    for (int c = 0; c < no_int_states; c++) gpu_check(m_gpu, atus_set_alpha(m_gpu, c, m_alpha.data()), "set_alpha");
    m_grid.h.dt = params->Get_dt();
    gpu_check(m_gpu, atus_set_time(m_gpu, m_grid.h.t), "set_time");
  }
  virtual ~CRT_Base() { atus_destroy(m_gpu); }

  double &Get_t() { return m_grid.h.t; }
  const double &Get_dt() const { return m_grid.h.dt; }
  long long &Get_dimX() { return m_grid.h.nDimX; }
  long long &Get_dimY() { return m_grid.h.nDimY; }
  long long &Get_dimZ() { return m_grid.h.nDimZ; }
  int64_t Get_No_Points() const { return m_grid.npts; }

  // Set_dt: store dt and rebuild the kinetic phases (CRT_shared.h:117-121)
  void Set_dt(double dt) {
    m_grid.h.dt = dt;
    gpu_check(m_gpu, atus_set_dt(m_gpu, dt), "set_dt");
  }

  double Get_Particle_Number(int comp = 0) {
    if (comp < 0 || comp > no_int_states) throw std::string("Error in Get_Particle_Number: comp out of bounds\n");
    double n = 0;
    gpu_check(m_gpu, atus_particle_number(m_gpu, comp, &n), "particle_number");
    return n;
  }

  void Setup_Momentum(CPoint<dim> p, int comp = 0) {
    if (comp < 0 || comp > no_int_states) throw std::string("Error in Setup_Momentum: comp out of bounds\n");
    gpu_check(m_gpu, atus_setup_momentum(m_gpu, comp, p.data()), "setup_momentum");
    m_host_valid = false;
  }
  void Expval_Position(CPoint<dim> &r, int comp = 0) {
    gpu_check(m_gpu, atus_expval_position(m_gpu, comp, r.data()), "expval_position");
  }
  void Expval_Momentum(CPoint<dim> &r, int comp = 0) {
    gpu_check(m_gpu, atus_expval_momentum(m_gpu, comp, r.data()), "expval_momentum");
  }

  void Save_Phi(const std::string &filename, int comp = 0) {
    sync_to_host();
    std::ofstream f(filename, std::ofstream::binary);
    f.write((const char *)&m_grid.h, sizeof(generic_header));
    f.write((const char *)m_fields[comp].data(), m_grid.npts * 16);
  }
  void Append_Phi(const std::string &filename, int comp = 0) {
    sync_to_host();
    std::ofstream f(filename, std::ofstream::binary | std::ofstream::app);
    if (f.fail()) {
      std::cout << "File " << filename << " could not be opened. Failbit: " << f.rdstate() << std::endl;
      exit(EXIT_FAILURE);
    }
    f.write((const char *)&m_grid.h, sizeof(generic_header));
    f.write((const char *)m_fields[comp].data(), m_grid.npts * 16);
  }

  void Set_custom_fct(StepFunction fct) { m_custom_fct = fct; }
  void Init_Potential() {
    for (auto &v : m_Potential) v.assign(m_grid.npts, 0.0);
    m_potenial_initialized = true;
    m_pot_dirty = true;
  }
  void Setup_Potential(int comp, int64_t index, double val) {
    if (!m_potenial_initialized) {
      std::cerr << "Potential not initialized. You forgot to invoke Init_Potential." << std::endl;
      throw std::string("Potential not initialized");
    }
    m_Potential[comp][index] = val;
    m_pot_dirty = true;
  }

  // The host copy of component c (downloaded on demand).
  fftw_complex *Getp2In(int c) {
    sync_to_host();
    return reinterpret_cast<fftw_complex *>(m_fields[c].data());
  }

  virtual void run_sequence() {
    char filename[1024];
    std::cout << "FYI: Found " << m_params->m_sequence.size() << " sequences." << std::endl;
    int seq_counter = 1;
    for (auto seq : m_params->m_sequence) {
      if (run_custom_sequence(seq)) continue;
      if (seq.name == "set_momentum") {
        set_momentum(seq);
        continue;
      }
      int Na, Nk;
      begin_sequence(seq, seq_counter, Na, Nk);
      for (int k = 0; k < no_int_states; k++) {
        snprintf(filename, sizeof filename, "Seq_%d_%d.bin", seq_counter, k + 1);
        std::remove(filename);
      }
      for (int i = 1; i <= Na; i++) {
        strang_block(seq, Nk);
        std::cout << "t = " << std::to_string(m_grid.h.t) << std::endl;
        if (seq.output_freq == each)
          for (int k = 0; k < no_int_states; k++) {
            snprintf(filename, sizeof filename, "%.3f_%d.bin", m_grid.h.t, k + 1);
            Save_Phi(filename, k);
          }
        if (seq.output_freq == packed)
          for (int k = 0; k < no_int_states; k++) {
            snprintf(filename, sizeof filename, "Seq_%d_%d.bin", seq_counter, k + 1);
            Append_Phi(filename, k);
          }
        if (seq.compute_pn_freq == each)
          for (int c = 0; c < no_int_states; c++)
            std::cout << "N[" << c << "] = " << Get_Particle_Number(c) << std::endl;
        if (seq.custom_freq == each && m_custom_fct != nullptr) call_host(m_custom_fct, seq);
      }
      if (seq.output_freq == last)
        for (int k = 0; k < no_int_states; k++) {
          snprintf(filename, sizeof filename, "%.3f_%d.bin", m_grid.h.t, k + 1);
          Save_Phi(filename, k);
        }
      if (seq.compute_pn_freq == last)
        for (int c = 0; c < no_int_states; c++)
          std::cout << "N[" << c << "] = " << Get_Particle_Number(c) << std::endl;
      if (seq.custom_freq == last && m_custom_fct != nullptr) call_host(m_custom_fct, seq);
      seq_counter++;
    }
  }

 protected:
  virtual bool run_custom_sequence(const sequence_item &) = 0;
  // Pulse amplitudes of the nk potential steps of the next block (1 without
  // an AMP_T); CRT_Base_IF evaluates AMP_T.
  virtual void pulse_amplitudes(const sequence_item &, int nk, std::vector<double> &F) { F.assign(nk, 1.0); }
  virtual void upload_step_parameters(const sequence_item &) {}

  static generic_header read_header(const std::string &filename) {
    std::ifstream f(filename, std::ifstream::binary);
    if (!f.is_open()) throw std::string("Could not open file " + filename + ".\n");
    generic_header h{};
    f.read((char *)&h, sizeof(generic_header));
    return h;
  }
  void load(const std::string &filename, int c) {
    std::ifstream f(filename, std::ifstream::binary);
    if (!f.is_open()) throw std::string("Could not open file " + filename + "\n");
    f.seekg(sizeof(generic_header), std::ifstream::beg);
    f.read((char *)m_fields[c].data(), m_grid.npts * 16);
  }

  void sync_to_host() {
    if (m_host_valid) return;
    for (int c = 0; c < no_int_states; c++) gpu_check(m_gpu, atus_download_psi(m_gpu, c, m_fields[c].data()), "download");
    m_host_valid = true;
  }
  void sync_to_device() {
    for (int c = 0; c < no_int_states; c++) gpu_check(m_gpu, atus_upload_psi(m_gpu, c, m_fields[c].data()), "upload");
    gpu_check(m_gpu, atus_set_time(m_gpu, m_grid.h.t), "set_time");
  }
  void flush_potential() {
    if (!m_pot_dirty) return;
    for (int c = 0; c < no_int_states; c++)
      gpu_check(m_gpu, atus_set_potential(m_gpu, c, m_potenial_initialized ? m_Potential[c].data() : nullptr),
                "set_potential");
    m_pot_dirty = false;
  }
  // A host step function sees and may change the host copy.
  void call_host(StepFunction f, sequence_item &seq) {
    sync_to_host();
    f(this, seq);
    sync_to_device();
  }

  void set_momentum(const sequence_item &seq) {
    std::vector<double> vec;
    std::string cur;
    for (char ch : seq.content + ",") {
      if (ch == ',') { vec.push_back(std::stod(cur)); cur.clear(); }
      else cur += ch;
    }
    CPoint<dim> P{};
    for (int i = 0; i < dim && i < (int)vec.size(); i++) P[i] = vec[i];
    Setup_Momentum(P, seq.comp);
    std::cout << "FYI: started new sequence " << seq.name << "\n";
    std::cout << "FYI: momentum set for component " << seq.comp << "\n";
  }

  // The preamble of a sequence (include/CRT_Base.h:737-768).
  void begin_sequence(const sequence_item &seq, int seq_counter, int &Na, int &Nk) {
    double max_duration = 0;
    for (double d : seq.duration)
      if (d > max_duration) max_duration = d;
    const int subN = int(max_duration / seq.dt);
    Nk = seq.Nk;
    Na = subN / seq.Nk;
    std::cout << "FYI: started new sequence " << seq.name << "\n";
    std::cout << "FYI: sequence no : " << seq_counter << "\n";
    std::cout << "FYI: duration    : " << max_duration << "\n";
    std::cout << "FYI: dt          : " << seq.dt << "\n";
    std::cout << "FYI: Na          : " << Na << "\n";
    std::cout << "FYI: Nk          : " << Nk << "\n";
    std::cout << "FYI: Na*Nk*dt    : " << double(Na * Nk) * seq.dt << "\n";
    if (double(Na * Nk) * seq.dt != max_duration) std::cout << "FYI: double(Na*Nk)*seq.dt != max_duration\n";
    if (Get_dt() != seq.dt) Set_dt(seq.dt);
    if (!m_gpu_steps.count(seq.name) && !m_map_stepfcts.count(seq.name)) {
      std::cerr << "Critical Error: Invalid squence name " << seq.name << "\n";
      exit(EXIT_FAILURE);
    }
  }

  // half, (V, full)^(Nk-1), V, half  (include/CRT_Base.h:776-786)
  void strang_block(sequence_item &seq, int Nk) {
    flush_potential();
    upload_step_parameters(seq);
    auto g = m_gpu_steps.find(seq.name);
    if (g != m_gpu_steps.end()) {
      std::vector<double> F;
      pulse_amplitudes(seq, Nk, F);
      gpu_check(m_gpu, atus_strang_block(m_gpu, Nk, g->second, F.data()), "strang_block");
      gpu_check(m_gpu, atus_get_time(m_gpu, &m_grid.h.t), "get_time");
      m_host_valid = false;
      return;
    }
    StepFunction f = m_map_stepfcts.at(seq.name);
    gpu_check(m_gpu, atus_ft_step(m_gpu, 1), "ft_step");
    gpu_check(m_gpu, atus_get_time(m_gpu, &m_grid.h.t), "get_time");
    m_host_valid = false;
    for (int j = 2; j <= Nk; j++) {
      call_host(f, seq);
      gpu_check(m_gpu, atus_ft_step(m_gpu, 0), "ft_step");
      gpu_check(m_gpu, atus_get_time(m_gpu, &m_grid.h.t), "get_time");
      m_host_valid = false;
    }
    call_host(f, seq);
    gpu_check(m_gpu, atus_ft_step(m_gpu, 1), "ft_step");
    gpu_check(m_gpu, atus_get_time(m_gpu, &m_grid.h.t), "get_time");
    m_host_valid = false;
  }

  ParameterHandler *m_params;
  Grid<dim> m_grid;
  atus_ctx *m_gpu = nullptr;
  std::array<double, no_int_states * no_int_states> m_gs{};
  CPoint<dim> m_alpha{};
  std::array<std::vector<double>, no_int_states> m_fields;
  bool m_host_valid = true;
  std::array<std::vector<double>, no_int_states> m_Potential;
  bool m_potenial_initialized = false, m_pot_dirty = false;
  std::map<std::string, int> m_gpu_steps;
  std::map<std::string, StepFunction> m_map_stepfcts;
  StepFunction m_custom_fct = nullptr;
};

// ============================================================== CRT_Base_IF
template <int dim, int no_int_states>
class CRT_Base_IF : public CRT_Base<dim, no_int_states> {
  using Base = CRT_Base<dim, no_int_states>;

 public:
  explicit CRT_Base_IF(ParameterHandler *params, int precision = ATUS_PREC_FP64) : Base(params, precision) {
    // include/CRT_Base_IF.h:120-129: freeprop and the numerical bragg / raman steps
    this->m_gpu_steps["freeprop"] = ATUS_STEP_NL_IF;
    this->m_gpu_steps["bragg"] = ATUS_STEP_NUMERICAL_BRAGG;
    this->m_gpu_steps["raman"] = ATUS_STEP_NUMERICAL_RAMAN;
    UpdateParams();
  }

  // CRT_Base_IF::run_sequence (include/CRT_Base_IF.h:638-946): as CRT_Base's,
  // plus the AMP_T envelope, Rabi sums and the chirp / phase scan.
  void run_sequence() override {
    char filename[1024];
    std::cout << "FYI: Found " << this->m_params->m_sequence.size() << " sequences." << std::endl;
    const int nrm = (int)m_rabi_momentum_list.size();
    if (nrm == 0) std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << std::endl;
    int seq_counter = 1;
    for (auto seq : this->m_params->m_sequence) {
      if (this->run_custom_sequence(seq)) {
        seq_counter++;
        continue;
      }
      if (seq.name == "set_momentum") {
        this->set_momentum(seq);
        continue;
      }
      double max_duration = 0;
      for (double d : seq.duration)
        if (d > max_duration) max_duration = d;
      const int subN = int(max_duration / seq.dt);
      const int Nk = seq.Nk;
      const int Na = subN / seq.Nk;
      std::cout << "FYI: started new sequence " << seq.name << "\n";
      std::cout << "FYI: sequence no : " << seq_counter << "\n";
      std::cout << "FYI: duration    : " << max_duration << "\n";
      std::cout << "FYI: dt          : " << seq.dt << "\n";
      std::cout << "FYI: Na          : " << Na << "\n";
      std::cout << "FYI: Nk          : " << Nk << "\n";
      std::cout << "FYI: Na*Nk*dt    : " << double(Na * Nk) * seq.dt << "\n";
      if (this->m_params->Has_simulation("AMP_T")) {
        std::cout << "FYI: Amp is      : " << this->m_params->Get_simulation("AMP_T") << "\n";
        amp_is_t = true;
      } else {
        std::cout << "FYI: Amp is      : 1" << std::endl;
        amp_is_t = false;
      }
      if (double(Na * Nk) * seq.dt != max_duration) std::cout << "FYI: double(Na*Nk)*seq.dt != max_duration\n";
      if (this->Get_dt() != seq.dt) this->Set_dt(seq.dt);
      if (!this->m_gpu_steps.count(seq.name) && !this->m_map_stepfcts.count(seq.name)) {
        std::cerr << "Critical Error: Invalid squence name " << seq.name << "\n";
        exit(EXIT_FAILURE);
      }
      if (seq.name == "freeprop") seq.no_of_chirps = 1;
      const double backup_t = this->m_grid.h.t;
      double backup_end_t = this->m_grid.h.t;
      for (int k = 0; k < no_int_states; k++) {
        snprintf(filename, sizeof filename, "Seq_%d_%d.bin", seq_counter, k + 1);
        std::remove(filename);
      }
      m_chirps_list.clear();
      std::vector<double> dw(std::max(seq.no_of_chirps, 2), 0.0), dphi(std::max(seq.no_of_chirps, 1), 0.0);
      if (seq.no_of_chirps > 1) {
        for (int k = 0; k < no_int_states; k++) {
          snprintf(filename, sizeof filename, "%.3f_%d.bin", this->Get_t(), k + 1);
          this->Save_Phi(filename, k);
        }
        dw[0] = seq.chirp_min;
        dw[1] = seq.chirp_max;
      } else {
        dw[0] = 0;
      }
      for (int s = 0; s < seq.no_of_chirps; ++s) {
        m_rabi_freq_list.clear();
        chirp_rate[0] = dw[s];
        if (seq.chirp_mode == 1) phase[0] = s * 2.0 * M_PI / (1.0 * seq.no_of_chirps);
        for (int i = 1; i <= Na; i++) {
          this->strang_block(seq, Nk);
          std::cout << "t = " << std::to_string(this->m_grid.h.t) << std::endl;
          if (seq.output_freq == each && s == 0)
            for (int k = 0; k < no_int_states; k++) {
              snprintf(filename, sizeof filename, "%.3f_%d.bin", this->Get_t(), k + 1);
              this->Save_Phi(filename, k);
            }
          if (seq.output_freq == packed && s == 0)
            for (int k = 0; k < no_int_states; k++) {
              snprintf(filename, sizeof filename, "Seq_%d_%d.bin", seq_counter, k + 1);
              this->Append_Phi(filename, k);
            }
          if (seq.compute_pn_freq == each)
            for (int c = 0; c < no_int_states; c++)
              std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
          if (seq.rabi_output_freq == each) compute_rabi_integrals();
          if (seq.custom_freq == each && this->m_custom_fct != nullptr) this->call_host(this->m_custom_fct, seq);
        }
        if (seq.output_freq == last && s == 0)
          for (int k = 0; k < no_int_states; k++) {
            snprintf(filename, sizeof filename, "%.3f_%d.bin", this->Get_t(), k + 1);
            this->Save_Phi(filename, k);
          }
        if (seq.no_of_chirps > 1 && s == 0) {
          backup_end_t = this->Get_t();
          for (int k = 0; k < no_int_states; k++) {
            snprintf(filename, sizeof filename, "%.3f_%d.bin", this->Get_t(), k + 1);
            this->Save_Phi(filename, k);
          }
        }
        if (seq.compute_pn_freq == last)
          for (int c = 0; c < no_int_states; c++)
            std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
        if (seq.custom_freq == last && this->m_custom_fct != nullptr) this->call_host(this->m_custom_fct, seq);
        if (seq.rabi_output_freq == last) {
          compute_rabi_integrals();
          std::cout << "Rabi output for timestep ";
          for (auto &row : m_rabi_freq_list) {
            std::cout << this->Get_t() << "\n";
            for (double v : row) std::cout << v << "\t";
            std::cout << std::endl;
          }
        }
        if (seq.rabi_output_freq == each) {
          snprintf(filename, sizeof filename, "Rabi_%d_%d.txt", seq_counter, s);
          Output_rabi_freq_list(filename, seq.Nk);
        }
        if (seq.no_of_chirps > 1) {
          if (nrm > 0) {
            compute_rabi_integrals();
            std::list<double> tmp = m_rabi_freq_list.back();
            if (seq.chirp_mode == 1) {
              tmp.push_front(phase[0]);
            } else {
              dphi[s] = tmp.front();
              tmp.push_front(chirp_rate[0]);
            }
            tmp.push_front(s);
            m_chirps_list.push_back(tmp);
          }
          if (s < seq.no_of_chirps - 1) {
            for (int k = 0; k < no_int_states; k++) {
              snprintf(filename, sizeof filename, "%.3f_%d.bin", backup_t, k + 1);
              reload(filename, k);
            }
            this->m_grid.h.t = backup_t;
            this->sync_to_device();
          }
          if (s > 0 && s < seq.no_of_chirps - 1) {
            dw[s + 1] = (dw[s] + dw[s - 1]) / 2;
            if (dphi[s] - dphi[s - 1] < 0) {
              dw[s] = dw[s - 1];
              dphi[s] = dphi[s - 1];
            }
          }
        }
      }
      if (seq.no_of_chirps > 1) {
        snprintf(filename, sizeof filename, "Chirp_%d.txt", seq_counter);
        Output_chirps_list(filename);
        for (int k = 0; k < no_int_states; k++) {
          snprintf(filename, sizeof filename, "%.3f_%d.bin", backup_end_t, k + 1);
          reload(filename, k);
        }
        this->m_grid.h.t = backup_end_t;
        this->sync_to_device();
      }
      seq_counter++;
    }
  }

 protected:
  // UpdateParams (include/CRT_Base_IF.h:144-168)
  void UpdateParams() {
    for (int i = 0; i < dim; i++) beta[i] = this->m_params->Get_VConstant("Beta", i);
    for (int i = 0; i < no_int_states; i++) DeltaL[i] = this->m_params->Get_VConstant("Delta_L", i);
    try {
      Amp[0] = this->m_params->Get_VConstant("Amp_1", 0);
      Amp[1] = this->m_params->Get_VConstant("Amp_1", 1);
      laser_k[0] = this->m_params->Get_Constant("laser_k");
      laser_dk[0] = this->m_params->Get_Constant("laser_dk");
      laser_domh[0] = this->m_params->Get_Constant("laser_domh");
      m_rabi_threshold = this->m_params->Get_Constant("rabi_threshold");
      chirp = this->m_params->Get_Constant("chirp");
    } catch (std::string &str) {
      std::cout << str << std::endl;
      exit(EXIT_FAILURE);
    }
  }

  void upload_step_parameters(const sequence_item &) override {
    atus_laser L{};
    for (int i = 0; i < dim; i++) L.beta[i] = beta[i];
    for (int i = 0; i < no_int_states; i++) L.DeltaL[i] = DeltaL[i];
    for (int i = 0; i < 2; i++) {
      L.Amp[i] = Amp[i];
      L.laser_k[i] = laser_k[i];
      L.laser_dk[i] = laser_dk[i];
      L.laser_domh[i] = laser_domh[i];
      L.phase[i] = phase[i];
      L.chirp_rate[i] = chirp_rate[i];
    }
    L.chirp = chirp;
    gpu_check(this->m_gpu, atus_set_laser(this->m_gpu, &L), "set_laser");
  }

  // AMP_T at t + dt/2 of every potential step of the coming block
  // (Amplitude_at_time, include/CRT_Base_IF.h:170-198).
  void pulse_amplitudes(const sequence_item &, int nk, std::vector<double> &F) override {
    F.assign(nk, 1.0);
    if (!amp_is_t) return;
    const double dt = this->Get_dt();
    double time = 0;
    Expr e;
    this->m_params->Setup_Parser(e);
    e.SetExpr(this->m_params->Get_simulation("AMP_T"));
    e.DefineVar("t", &time);
    double t = this->m_grid.h.t + 0.5 * dt;  // after the leading half step
    for (int j = 0; j < nk; j++) {
      time = t + 0.5 * dt;
      F[j] = e.Eval();
      t += dt;
    }
  }

  void compute_rabi_integrals() {
    const int n = (int)m_rabi_momentum_list.size();
    if (n == 0) {
      std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << std::endl;
      return;
    }
    std::vector<double> k0, res(n);
    for (auto &p : m_rabi_momentum_list)
      for (int a = 0; a < dim; a++) k0.push_back(p[a]);
    gpu_check(this->m_gpu, atus_rabi_integrals(this->m_gpu, k0.data(), n, m_rabi_threshold, res.data()), "rabi");
    m_rabi_freq_list.push_back(std::list<double>(res.begin(), res.end()));
  }

  void Output_rabi_freq_list(const std::string &filename, long long Nk) {
    std::ofstream txt(filename);
    double t = 0;
    txt << "# time \t";
    for (auto &p : m_rabi_momentum_list) {
      for (int a = 0; a < dim; a++) txt << p[a] << ((a == dim - 1) ? "" : ",");
      txt << "\t";
    }
    txt << std::endl;
    for (auto &row : m_rabi_freq_list) {
      txt << t << "\t";
      for (double v : row) txt << v << "\t";
      txt << std::endl;
      t += this->m_grid.h.dt * double(Nk);
    }
  }
  void Output_chirps_list(const std::string &filename) {
    std::ofstream txt(filename);
    txt << "# Step \t Chirp \t ";
    for (auto &p : m_rabi_momentum_list) {
      for (int a = 0; a < dim; a++) txt << p[a] << ((a == dim - 1) ? "" : ",");
      txt << "\t";
    }
    txt << std::endl;
    for (auto &row : m_chirps_list) {
      for (double v : row) {
        txt.precision(8);
        txt << v << "\t";
      }
      txt << std::endl;
    }
  }
  void reload(const std::string &filename, int k) {
    this->load(filename, k);
    this->m_host_valid = true;
  }

  CPoint<dim> beta{};
  std::array<double, no_int_states> DeltaL{};
  std::array<double, 2> Amp{}, laser_k{}, laser_dk{}, laser_domh{}, phase{}, chirp_rate{};
  double chirp = 0;
  bool amp_is_t = false;
  double m_rabi_threshold = 0;
  std::vector<CPoint<dim>> m_rabi_momentum_list;
  std::list<std::list<double>> m_rabi_freq_list, m_chirps_list;
};

// ============================================================== CRT_Base_IF_2
// Two species of two internal states each (include/CRT_Base_2.h,
// include/CRT_Base_IF_2.h): components [0, n/2) are species 1 with Alpha_1,
// Beta and the laser constants, [n/2, n) species 2 with Alpha_2, Beta_2 and the
// *_2 constants.  "freeprop" is CRT_Base_IF_2::Do_NL_Step (GPU kind
// ATUS_STEP_NL_IF_2); "freeprop_lin" only takes the kinetic steps
// (CRT_Base_2.h:283-286 is empty).
template <int dim, int no_int_states>
class CRT_Base_IF_2 : public CRT_Base<dim, no_int_states> {
  using Base = CRT_Base<dim, no_int_states>;

 public:
  explicit CRT_Base_IF_2(ParameterHandler *params, int precision = ATUS_PREC_FP64) : Base(params, precision) {
    // CRT_Base_2's constructor reads Alpha_2 after Init() as it reads Alpha_1
    // (include/CRT_Base_2.h:125-129): the tables follow at the next Set_dt
    for (int i = 0; i < dim; i++) m_alpha2[i] = this->m_params->Get_VConstant("Alpha_2", i);
    for (int c = no_int_states / 2; c < no_int_states; c++)
      gpu_check(this->m_gpu, atus_set_alpha(this->m_gpu, c, m_alpha2.data()), "set_alpha");
    this->m_gpu_steps["freeprop"] = ATUS_STEP_NL_IF_2;
    this->m_map_stepfcts["freeprop_lin"] = &Do_Nothing;
    UpdateParams();
  }

  // CRT_Base_IF_2::run_sequence (include/CRT_Base_IF_2.h:420-593).
  void run_sequence() override {
    char filename[1024], filename2[1024];
    std::cout << "FYI: Found " << this->m_params->m_sequence.size() << " sequences." << std::endl;
    const int nrm = (int)m_rabi_momentum_list.size();
    if (nrm == 0) std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << std::endl;
    int seq_counter = 1;
    for (auto seq : this->m_params->m_sequence) {
      if (this->run_custom_sequence(seq)) continue;
      if (seq.name == "set_momentum") {
        this->set_momentum(seq);
        continue;
      }
      double max_duration = 0;
      for (double d : seq.duration)
        if (d > max_duration) max_duration = d;
      const int subN = int(max_duration / seq.dt);
      const int Nk = seq.Nk;
      const int Na = subN / seq.Nk;
      seq.time = this->Get_t();
      std::cout << "FYI: started new sequence " << seq.name << "\n";
      std::cout << "FYI: sequence no : " << seq_counter << "\n";
      std::cout << "FYI: duration    : " << max_duration << "\n";
      std::cout << "FYI: dt          : " << seq.dt << "\n";
      std::cout << "FYI: Na          : " << Na << "\n";
      std::cout << "FYI: Nk          : " << Nk << "\n";
      std::cout << "FYI: Na*Nk*dt    : " << double(Na * Nk) * seq.dt << "\n";
      if (double(Na * Nk) * seq.dt != max_duration) std::cout << "FYI: double(Na*Nk)*seq.dt != max_duration\n";
      if (this->Get_dt() != seq.dt) this->Set_dt(seq.dt);
      if (!this->m_gpu_steps.count(seq.name) && !this->m_map_stepfcts.count(seq.name)) {
        std::cerr << "Critical Error: Invalid squence name " << seq.name << "\n";
        exit(EXIT_FAILURE);
      }
      if (seq.name == "freeprop") seq.no_of_chirps = 1;
      const double backup_t = this->m_grid.h.t;
      m_chirps_list.clear();
      for (int s = 0; s < seq.no_of_chirps; ++s) {
        m_rabi_freq_list.clear();
        m_rabi_freq_list2.clear();
        chirp_rate[0] = 0.0;
        for (int i = 1; i <= Na; i++) {
          this->strang_block(seq, Nk);
          std::cout << "t = " << std::to_string(this->m_grid.h.t) << std::endl;
          if (seq.output_freq == each) save_all();
          if (seq.compute_pn_freq == each)
            for (int c = 0; c < no_int_states; c++)
              std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
          if (seq.rabi_output_freq == each) compute_rabi_integrals();
          if (seq.custom_freq == each && this->m_custom_fct != nullptr) this->call_host(this->m_custom_fct, seq);
        }
        if (seq.output_freq == last) save_all();
        if (seq.compute_pn_freq == last)
          for (int c = 0; c < no_int_states; c++)
            std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
        if (seq.custom_freq == last && this->m_custom_fct != nullptr) this->call_host(this->m_custom_fct, seq);
        if (seq.rabi_output_freq == last) {
          compute_rabi_integrals();
          std::cout << "Spezie 1" << std::endl;
          std::cout << "Rabi output for timestep ";
          for (auto &row : m_rabi_freq_list) {
            std::cout << this->Get_t() << "\n";
            for (double v : row) std::cout << v << "\t";
            std::cout << std::endl;
          }
          std::cout << "Spezie 2" << std::endl;
          for (auto &row : m_rabi_freq_list2) {
            std::cout << this->Get_t() << "\n";
            for (double v : row) std::cout << v << "\t";
            std::cout << std::endl;
          }
        }
        if (seq.rabi_output_freq == each) {
          snprintf(filename, sizeof filename, "Spezie_%d_Rabi_%d_%d.txt", 1, seq_counter, s);
          snprintf(filename2, sizeof filename2, "Spezie_%d_Rabi_%d_%d.txt", 2, seq_counter, s);
          Output_rabi_freq_list(filename, filename2, seq.Nk);
        }
        if (seq.no_of_chirps > 1 && nrm > 0) {
          compute_rabi_integrals();
          std::list<double> tmp = m_rabi_freq_list.back();
          tmp.push_front(chirp_rate[0]);
          tmp.push_front(s);
          m_chirps_list.push_back(tmp);
        }
        // the scan restarts from the files of the sequence's start time; a
        // file that does not open leaves the fields as they are
        if (seq.no_of_chirps > 1 && s < seq.no_of_chirps - 1) {
          this->sync_to_host();
          for (int k = 0; k < no_int_states; k++) {
            snprintf(filename, sizeof filename, "%.3f_%d.bin", backup_t, k + 1);
            std::ifstream f(filename, std::ifstream::binary);
            if (!f.is_open()) continue;
            f.seekg(sizeof(generic_header), std::ifstream::beg);
            f.read((char *)this->m_fields[k].data(), this->m_grid.npts * 16);
          }
          this->m_grid.h.t = backup_t;
          this->sync_to_device();
        }
      }
      if (seq.no_of_chirps > 1) {
        snprintf(filename, sizeof filename, "Chirp_%d.txt", seq_counter);
        Output_chirps_list(filename);
      }
      seq_counter++;
    }
  }

 protected:
  static void Do_Nothing(void *, sequence_item &) {}

  // UpdateParams (include/CRT_Base_IF_2.h:80-113); phase, phase2 and
  // chirp_rate2 are never set by the reference and stay 0.
  void UpdateParams() {
    for (int i = 0; i < dim; i++) {
      beta[i] = this->m_params->Get_VConstant("Beta", i);
      beta2[i] = this->m_params->Get_VConstant("Beta_2", i);
    }
    for (int i = 0; i < no_int_states; i++) DeltaL[i] = this->m_params->Get_VConstant("Delta_L", i);
    try {
      Amp[0] = this->m_params->Get_VConstant("Amp_1", 0);
      Amp[1] = this->m_params->Get_VConstant("Amp_1", 1);
      Amp2[0] = this->m_params->Get_VConstant("Amp_2", 0);
      Amp2[1] = this->m_params->Get_VConstant("Amp_2", 1);
      laser_k[0] = this->m_params->Get_Constant("laser_k");
      laser_k2[0] = this->m_params->Get_Constant("laser_k_2");
      laser_dk[0] = this->m_params->Get_Constant("laser_dk");
      laser_dk2[0] = this->m_params->Get_Constant("laser_dk_2");
      laser_domh[0] = this->m_params->Get_Constant("laser_domh");
      laser_domh2[0] = this->m_params->Get_Constant("laser_domh_2");
      m_rabi_threshold = this->m_params->Get_Constant("rabi_threshold");
    } catch (std::string &str) {
      std::cout << str << std::endl;
    }
  }

  // Both species' lasers and the pulse windows of the sequence.  bragg_ds
  // reads seq.duration[0] and [1] (bragg_ds.cpp:122-125); a sequence with a
  // single duration uses it for both species.
  void upload_step_parameters(const sequence_item &seq) override {
    atus_laser L{}, L2{};
    for (int i = 0; i < dim; i++) {
      L.beta[i] = beta[i];
      L2.beta[i] = beta2[i];
    }
    for (int i = 0; i < no_int_states; i++) L.DeltaL[i] = DeltaL[i];
    for (int i = 0; i < 2; i++) {
      L.Amp[i] = Amp[i];
      L.laser_k[i] = laser_k[i];
      L.laser_dk[i] = laser_dk[i];
      L.laser_domh[i] = laser_domh[i];
      L.phase[i] = phase[i];
      L.chirp_rate[i] = chirp_rate[i];
      L2.Amp[i] = Amp2[i];
      L2.laser_k[i] = laser_k2[i];
      L2.laser_dk[i] = laser_dk2[i];
      L2.laser_domh[i] = laser_domh2[i];
      L2.phase[i] = phase2[i];
      L2.chirp_rate[i] = chirp_rate2[i];
    }
    gpu_check(this->m_gpu, atus_set_laser(this->m_gpu, &L), "set_laser");
    gpu_check(this->m_gpu, atus_set_laser2(this->m_gpu, &L2), "set_laser2");
    double dur[2] = {HUGE_VAL, HUGE_VAL};
    if (!seq.duration.empty()) dur[0] = dur[1] = seq.duration[0];
    if (seq.duration.size() > 1) dur[1] = seq.duration[1];
    gpu_check(this->m_gpu, atus_set_pulse_windows(this->m_gpu, seq.time, dur), "set_pulse_windows");
  }

  void save_all() {
    char filename[1024];
    for (int k = 0; k < no_int_states; k++) {
      snprintf(filename, sizeof filename, "%.3f_%d.bin", this->Get_t(), k + 1);
      this->Save_Phi(filename, k);
    }
  }

  // CRT_Base_IF_2::compute_rabi_integrals (include/CRT_Base_IF_2.h:115-210):
  // species 1 on component 0, species 2 on component no_int_states/2.
  void compute_rabi_integrals() {
    const int n = (int)m_rabi_momentum_list.size(), m = (int)m_rabi_momentum_list2.size();
    if (n == 0 || m == 0) {
      std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << std::endl;
      return;
    }
    std::vector<double> k0, k02, res(n), res2(m);
    for (auto &p : m_rabi_momentum_list)
      for (int a = 0; a < dim; a++) k0.push_back(p[a]);
    for (auto &p : m_rabi_momentum_list2)
      for (int a = 0; a < dim; a++) k02.push_back(p[a]);
    gpu_check(this->m_gpu, atus_rabi_integrals_comp(this->m_gpu, 0, k0.data(), n, m_rabi_threshold, res.data()),
              "rabi");
    gpu_check(this->m_gpu,
              atus_rabi_integrals_comp(this->m_gpu, no_int_states / 2, k02.data(), m, m_rabi_threshold, res2.data()),
              "rabi");
    m_rabi_freq_list.push_back(std::list<double>(res.begin(), res.end()));
    m_rabi_freq_list2.push_back(std::list<double>(res2.begin(), res2.end()));
  }

  static void write_rabi(const std::string &filename, const std::vector<CPoint<dim>> &pts,
                         const std::list<std::list<double>> &rows, double dt_out) {
    std::ofstream txt(filename);
    double t = 0;
    txt << "# time \t";
    for (auto &p : pts) {
      for (int a = 0; a < dim; a++) txt << p[a] << ((a == dim - 1) ? "" : ",");
      txt << "\t";
    }
    txt << std::endl;
    for (auto &row : rows) {
      txt << t << "\t";
      for (double v : row) txt << v << "\t";
      txt << std::endl;
      t += dt_out;
    }
  }
  void Output_rabi_freq_list(const std::string &filename, const std::string &filename2, long long Nk) {
    write_rabi(filename, m_rabi_momentum_list, m_rabi_freq_list, this->m_grid.h.dt * double(Nk));
    write_rabi(filename2, m_rabi_momentum_list2, m_rabi_freq_list2, this->m_grid.h.dt * double(Nk));
  }
  void Output_chirps_list(const std::string &filename) {
    std::ofstream txt(filename);
    txt << "# Step \t Chirp \t ";
    for (auto &p : m_rabi_momentum_list) {
      for (int a = 0; a < dim; a++) txt << p[a] << ((a == dim - 1) ? "" : ",");
      txt << "\t";
    }
    txt << std::endl;
    for (auto &row : m_chirps_list) {
      for (double v : row) txt << v << "\t";
      txt << std::endl;
    }
  }

  CPoint<dim> m_alpha2{}, beta{}, beta2{};
  std::array<double, no_int_states> DeltaL{};
  std::array<double, 2> Amp{}, Amp2{}, laser_k{}, laser_k2{}, laser_dk{}, laser_dk2{}, laser_domh{}, laser_domh2{},
      phase{}, phase2{}, chirp_rate{}, chirp_rate2{};
  double m_rabi_threshold = 0;
  std::vector<CPoint<dim>> m_rabi_momentum_list, m_rabi_momentum_list2;
  std::list<std::list<double>> m_rabi_freq_list, m_rabi_freq_list2, m_chirps_list;
};

// ============================================================== CSOB_Base
template <int dim, int no_wf>
class CSOB_Base {
 public:
  explicit CSOB_Base(ParameterHandler *params) : m_params(params) {
    // header from ALGORITHM (include/CSOB_Base.h:101-168)
    generic_header &h = m_grid.h;
    h = generic_header{};
    h.nself = sizeof(generic_header);
    h.bAtom = 1;
    h.bComplex = 1;
    h.nDatatyp = 16;
    h.nDims = dim;
    h.dt = 0.01;
    h.nDimX = params->Get_NX();
    h.nDimY = dim >= 2 ? params->Get_NY() : 1;
    h.nDimZ = dim >= 3 ? params->Get_NZ() : 1;
    h.xMax = params->Get_xMax();
    h.xMin = params->Get_xMin();
    h.dx = std::fabs(h.xMax - h.xMin) / double(h.nDimX);
    h.dkx = 2 * M_PI / std::fabs(h.xMax - h.xMin);
    if (dim >= 2) {
      h.yMax = params->Get_yMax();
      h.yMin = params->Get_yMin();
      h.dy = std::fabs(h.yMax - h.yMin) / double(h.nDimY);
      h.dky = 2 * M_PI / std::fabs(h.yMax - h.yMin);
    }
    if (dim >= 3) {
      h.zMax = params->Get_zMax();
      h.zMin = params->Get_zMin();
      h.dz = std::fabs(h.zMax - h.zMin) / double(h.nDimZ);
      h.dkz = 2 * M_PI / std::fabs(h.zMax - h.zMin);
    }
    m_grid.setup();
    for (int i = 0; i < no_wf; i++)
      for (int j = 0; j < no_wf; j++)
        m_gs[j + no_wf * i] = params->Get_VConstant("GS_" + std::to_string(i + 1), j) *
                              std::sqrt(params->Get_VConstant("N", i)) * std::sqrt(params->Get_VConstant("N", j));
    for (int i = 0; i < no_wf; i++) m_alpha[i] = params->Get_VConstant("Alpha_" + std::to_string(i + 1), 0);
    h.dt = params->Get_dt();
    m_epsilon = params->Get_Constant("epsilon");
    m_stepsize = params->Get_Constant("stepsize");
    for (int i = 0; i < no_wf; i++) {
      m_Psi[i].assign(2 * m_grid.npts, 0.0);
      m_Potential[i].assign(m_grid.npts, 0.0);
    }
    const atus_grid g = m_grid.abi();
    gpu_check(nullptr, atus_create(&g, no_wf, ATUS_PREC_FP64, &m_gpu), "atus_create");
    gpu_check(m_gpu, atus_set_gs(m_gpu, m_gs.data()), "set_gs");
    gpu_check(m_gpu, atus_sob_init(m_gpu, m_alpha.data(), m_stepsize), "sob_init");
  }
  virtual ~CSOB_Base() { atus_destroy(m_gpu); }

  double Get_Particle_Number(int comp = 0) {
    double n = 0;
    gpu_check(m_gpu, atus_particle_number(m_gpu, comp, &n), "particle_number");
    return n;
  }

  // CSOB_Base::run (include/CSOB_Base.h:426-505), with its console output.
  void run() {
    for (int i = 0; i < no_wf; i++) {
      gpu_check(m_gpu, atus_upload_psi(m_gpu, i, m_Psi[i].data()), "upload");
      gpu_check(m_gpu, atus_set_potential(m_gpu, i, m_Potential[i].data()), "set_potential");
    }
    gpu_check(m_gpu, atus_sob_renormalize(m_gpu), "renormalize");
    const bool quiet = std::getenv("ATUS_SOB_QUIET") != nullptr;
    int counter = 0;
    do {
      double N[ATUS_MAX_COMP];
      gpu_check(m_gpu, atus_sob_iterate(m_gpu, 1, &m_res_tot, N), "sob_iterate");
      if (!quiet) {
        bool brenorm = false;
        for (int i = 0; i < no_wf; i++) {
          if (std::fabs(N[i] - 1) > 1e-5) brenorm = true;
          std::cout << "N[" << i << "] = " << N[i] << std::endl;
        }
        printf("brenorm = %s\n", brenorm ? "true" : "false");
        std::cout << "--- " << counter << std::endl;
        std::cout << "res " << m_res_tot << std::endl;
      }
      counter++;
    } while (m_res_tot > m_epsilon);
    m_iterations = counter;
    for (int i = 0; i < no_wf; i++) gpu_check(m_gpu, atus_download_psi(m_gpu, i, m_Psi[i].data()), "download");
  }

  void Save(const std::vector<std::string> &filenames, bool rescale = false) {
    for (int i = 0; i < no_wf; i++) {
      if (rescale) {
        const double fak = std::sqrt(m_params->Get_VConstant("N", i));
        for (auto &v : m_Psi[i]) v *= fak;
      }
      std::cout << filenames[i] << std::endl;
      write(m_Psi[i], filenames[i]);
    }
  }
  void Save_Zero() {
    std::vector<double> z(2 * m_grid.npts, 0.0);
    std::cout << "zero.bin" << std::endl;
    write(z, "zero.bin");
  }
  int Iterations() const { return m_iterations; }
  double Residual() const { return m_res_tot; }

 protected:
  void write(const std::vector<double> &data, const std::string &filename) {
    std::ofstream f(filename, std::ofstream::binary);
    f.write((const char *)&m_grid.h, sizeof(generic_header));
    f.write((const char *)data.data(), m_grid.npts * 16);
  }

  ParameterHandler *m_params;
  Grid<dim> m_grid;
  atus_ctx *m_gpu = nullptr;
  std::array<double, no_wf * no_wf> m_gs{};
  std::array<double, no_wf> m_alpha{};
  double m_epsilon = 0, m_stepsize = 0, m_res_tot = 0;
  int m_iterations = 0;
  std::array<std::vector<double>, no_wf> m_Psi, m_Potential;
};

}  // namespace atus
