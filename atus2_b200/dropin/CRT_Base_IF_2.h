// CRT_Base_IF_2.h (drop-in) -- interferometry with two species, with the
// interface of ATUS-2's template <class T, int dim, int no_int_states> class
// CRT_Base_IF_2 (include/CRT_Base_IF_2.h:41-81): species 1 on components
// [0, n/2) with Beta, Amp_1, laser_k, laser_dk, laser_domh, species 2 on
// [n/2, n) with the *_2 constants; Rabi sums per species; freeprop as
// CRT_Base_IF_2::Do_NL_Step.  phase, phase2 and chirp_rate2 are never set by
// the reference and stay 0.
//
// GPU step tags: "freeprop" (both species' g|psi|^2 + beta x - DeltaL) and,
// for four components, "bragg_ad" -- the per-species two-level step of the
// bragg_ds program (source/interferometry/src/bragg_ds.cpp:111-322) with its
// pulse windows (seq.time, seq.duration[0..1]).
#ifndef ATUS_DROPIN_CRT_BASE_IF_2_H
#define ATUS_DROPIN_CRT_BASE_IF_2_H

#include <cmath>
#include <list>
#include <string>
#include <vector>

#include "CRT_Base_2.h"
#include "muParser.h"

using namespace std;

template <class T, int dim, int no_int_states>
class CRT_Base_IF_2 : public CRT_Base_2<T, dim, no_int_states> {
 public:
  CRT_Base_IF_2(ParameterHandler *params) : CRT_Base_2<T, dim, no_int_states>(params) {
    DeltaL.fill(0);
    for (auto *a : {&Amp, &Amp2, &laser_k, &laser_k2, &laser_dk, &laser_dk2, &laser_domh, &laser_domh2, &phase,
                    &phase2, &chirp_rate, &chirp_rate2})
      a->fill(0);
    this->m_map_stepfcts["freeprop"] = &Do_NL_Step_Wrapper;
    this->m_gpu_steps["freeprop"] = ATUS_STEP_NL_IF_2;
    if (no_int_states == 4) this->m_gpu_steps["bragg_ad"] = ATUS_STEP_BRAGG_DS_AD;
    m_workspace = nullptr;
    UpdateParams();
  }
  virtual ~CRT_Base_IF_2() {}

  void run_sequence();

 protected:
  using CRT_Base_2<T, dim, no_int_states>::m_header;
  using CRT_Base_2<T, dim, no_int_states>::m_params;
  using CRT_Base_2<T, dim, no_int_states>::m_fields;
  using CRT_Base_2<T, dim, no_int_states>::m_custom_fct;
  using CRT_shared::m_no_of_pts;

  CPoint<dim> beta, beta2;
  std::array<double, no_int_states> DeltaL;
  std::array<double, 2> Amp, Amp2, laser_k, laser_k2, laser_dk, laser_dk2, laser_domh, laser_domh2, phase, phase2,
      chirp_rate, chirp_rate2;

  static void Do_NL_Step_Wrapper(void *ptr, sequence_item &) { static_cast<CRT_Base_IF_2 *>(ptr)->Do_NL_Step(); }
  // CRT_Base_IF_2::Do_NL_Step (include/CRT_Base_IF_2.h:212-262) on the GPU
  void Do_NL_Step() {
    upload_lasers(nullptr);
    this->gpu_before();
    atus_check(this->m_gpu, atus_nl_step(this->m_gpu, ATUS_STEP_NL_IF_2, 1.0), "nl_step");
    this->gpu_after();
  }
  // UpdateParams (include/CRT_Base_IF_2.h:96-113)
  void UpdateParams() {
    for (int i = 0; i < dim; i++) {
      beta[i] = m_params->Get_VConstant("Beta", i);
      beta2[i] = m_params->Get_VConstant("Beta_2", i);
    }
    for (int i = 0; i < no_int_states; i++) DeltaL[i] = m_params->Get_VConstant("Delta_L", i);
    try {
      Amp[0] = m_params->Get_VConstant("Amp_1", 0);
      Amp[1] = m_params->Get_VConstant("Amp_1", 1);
      Amp2[0] = m_params->Get_VConstant("Amp_2", 0);
      Amp2[1] = m_params->Get_VConstant("Amp_2", 1);
      laser_k[0] = m_params->Get_Constant("laser_k");
      laser_k2[0] = m_params->Get_Constant("laser_k_2");
      laser_dk[0] = m_params->Get_Constant("laser_dk");
      laser_dk2[0] = m_params->Get_Constant("laser_dk_2");
      laser_domh[0] = m_params->Get_Constant("laser_domh");
      laser_domh2[0] = m_params->Get_Constant("laser_domh_2");
      m_rabi_threshold = m_params->Get_Constant("rabi_threshold");
    } catch (std::string &str) {
      cout << str << endl;
    }
  }
  void Output_rabi_freq_list(string filename, string filename2, const long long Nk) {
    write_rabi(filename, m_rabi_momentum_list, m_rabi_freq_list, m_header.dt * double(Nk));
    write_rabi(filename2, m_rabi_momentum_list2, m_rabi_freq_list2, m_header.dt * double(Nk));
  }
  void Output_chirps_list(string filename) {
    ofstream txt(filename);
    txt << "# Step \t Chirp \t ";
    for (auto &p : m_rabi_momentum_list) txt << p << "\t";
    txt << endl;
    for (auto &row : m_chirps_list) {
      for (double v : row) txt << v << "\t";
      txt << endl;
    }
  }

  virtual bool run_custom_sequence(const sequence_item &) = 0;

  fftw_complex *m_workspace;
  double m_rabi_threshold = 0;
  vector<CPoint<dim>> m_rabi_momentum_list;
  vector<CPoint<dim>> m_rabi_momentum_list2;
  list<list<double>> m_rabi_freq_list;
  list<list<double>> m_rabi_freq_list2;
  list<list<double>> m_chirps_list;

  // CRT_Base_IF_2::compute_rabi_integrals (include/CRT_Base_IF_2.h:115-210):
  // species 1 on component 0, species 2 on component no_int_states/2
  void compute_rabi_integrals() {
    const int n = (int)m_rabi_momentum_list.size(), m = (int)m_rabi_momentum_list2.size();
    if (n == 0 || m == 0) {
      std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << endl;
      return;
    }
    std::vector<double> k0, k02, res(n), res2(m);
    for (auto &p : m_rabi_momentum_list)
      for (int a = 0; a < dim; a++) k0.push_back(p[a]);
    for (auto &p : m_rabi_momentum_list2)
      for (int a = 0; a < dim; a++) k02.push_back(p[a]);
    this->gpu_before();
    atus_check(this->m_gpu, atus_rabi_integrals_comp(this->m_gpu, 0, k0.data(), n, m_rabi_threshold, res.data()),
               "rabi");
    atus_check(this->m_gpu,
               atus_rabi_integrals_comp(this->m_gpu, no_int_states / 2, k02.data(), m, m_rabi_threshold, res2.data()),
               "rabi");
    this->gpu_after(false);
    m_rabi_freq_list.push_back(list<double>(res.begin(), res.end()));
    m_rabi_freq_list2.push_back(list<double>(res2.begin(), res2.end()));
  }

  // ---- GPU side
  // both species' lasers and, with a sequence, bragg_ds's pulse windows: it
  // reads seq.duration[0] and [1] (bragg_ds.cpp:122-125); a sequence with a
  // single duration uses it for both species
  void upload_lasers(const sequence_item *seq) {
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
    atus_check(this->m_gpu, atus_set_laser(this->m_gpu, &L), "set_laser");
    atus_check(this->m_gpu, atus_set_laser2(this->m_gpu, &L2), "set_laser2");
    if (seq) {
      double dur[2] = {HUGE_VAL, HUGE_VAL};
      if (!seq->duration.empty()) dur[0] = dur[1] = seq->duration[0];
      if (seq->duration.size() > 1) dur[1] = seq->duration[1];
      atus_check(this->m_gpu, atus_set_pulse_windows(this->m_gpu, seq->time, dur), "set_pulse_windows");
    }
  }
  void upload_step_parameters(const sequence_item &seq) override { upload_lasers(&seq); }

  static void write_rabi(const std::string &filename, const vector<CPoint<dim>> &pts, const list<list<double>> &rows,
                         double dt_out) {
    ofstream txt(filename);
    double t = 0;
    txt << "# time \t";
    for (auto &p : pts) txt << p << "\t";
    txt << endl;
    for (auto &row : rows) {
      txt << t << "\t";
      for (double v : row) txt << v << "\t";
      txt << endl;
      t += dt_out;
    }
  }
  void save_all() { this->output_point("%.3f_%d.bin", false); }
};

// CRT_Base_IF_2::run_sequence (include/CRT_Base_IF_2.h:420-593)
template <class T, int dim, int no_int_states>
void CRT_Base_IF_2<T, dim, no_int_states>::run_sequence() {
  char filename[1024], filename2[1024];
  std::cout << "FYI: Found " << m_params->m_sequence.size() << " sequences." << std::endl;
  const int nrm = (int)m_rabi_momentum_list.size();
  if (nrm == 0) std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << endl;
  StepFunction half_fct = nullptr, full_fct = nullptr;
  try {
    half_fct = this->m_map_stepfcts.at("half_step");
    full_fct = this->m_map_stepfcts.at("full_step");
  } catch (const std::out_of_range &oor) {
    std::cerr << "Critical Error: Invalid fct ptr to ft_half_step or ft_full_step ()" << oor.what() << ")\n";
    exit(EXIT_FAILURE);
  }
  this->m_pot_dirty = true;
  int seq_counter = 1;
  for (auto seq : m_params->m_sequence) {
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
    this->print_sequence(seq, seq_counter, max_duration, Na, Nk);
    if (double(Na * Nk) * seq.dt != max_duration) std::cout << "FYI: double(Na*Nk)*seq.dt != max_duration\n";
    if (this->Get_dt() != seq.dt) this->Set_dt(seq.dt);
    StepFunction step_fct = this->step_function(seq.name);
    if (seq.name == "freeprop") seq.no_of_chirps = 1;
    const double backup_t = m_header.t;
    m_chirps_list.clear();
    for (int s = 0; s < seq.no_of_chirps; ++s) {
      m_rabi_freq_list.clear();
      m_rabi_freq_list2.clear();
      chirp_rate[0] = 0.0;
      for (int i = 1; i <= Na; i++) {
        // with Rabi output each block, both species' sums come out of the
        // block's last kinetic pass where it runs fused on the GPU
        bool rabi_done = false;
        if (seq.rabi_output_freq == freq::each && nrm > 0 && !m_rabi_momentum_list2.empty()) {
          std::vector<std::vector<double>> sums;
          rabi_done = this->strang_block_rabi(seq, Nk, step_fct, half_fct, full_fct, {0, no_int_states / 2},
                                              {&m_rabi_momentum_list, &m_rabi_momentum_list2}, m_rabi_threshold,
                                              sums);
          if (rabi_done) {
            m_rabi_freq_list.push_back(list<double>(sums[0].begin(), sums[0].end()));
            m_rabi_freq_list2.push_back(list<double>(sums[1].begin(), sums[1].end()));
          }
        } else {
          this->strang_block(seq, Nk, step_fct, half_fct, full_fct);
        }
        std::cout << "t = " << to_string(m_header.t) << std::endl;
        if (seq.output_freq == freq::each) save_all();
        if (seq.compute_pn_freq == freq::each)
          for (int c = 0; c < no_int_states; c++)
            std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
        if (seq.rabi_output_freq == freq::each && !rabi_done) compute_rabi_integrals();
        if (seq.custom_freq == freq::each && m_custom_fct != nullptr) {
          this->finish_output();
          (*m_custom_fct)(this, seq);
        }
      }
      if (seq.output_freq == freq::last) save_all();
      if (seq.compute_pn_freq == freq::last)
        for (int c = 0; c < no_int_states; c++)
          std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
      if (seq.custom_freq == freq::last && m_custom_fct != nullptr) {
        this->finish_output();
        (*m_custom_fct)(this, seq);
      }
      if (seq.rabi_output_freq == freq::last) {
        compute_rabi_integrals();
        cout << "Spezie 1" << endl;
        cout << "Rabi output for timestep ";
        for (auto &row : m_rabi_freq_list) {
          cout << this->Get_t() << "\n";
          for (double v : row) cout << v << "\t";
          cout << endl;
        }
        cout << "Spezie 2" << endl;
        for (auto &row : m_rabi_freq_list2) {
          cout << this->Get_t() << "\n";
          for (double v : row) cout << v << "\t";
          cout << endl;
        }
      }
      if (seq.rabi_output_freq == freq::each) {
        snprintf(filename, sizeof filename, "Spezie_%d_Rabi_%d_%d.txt", 1, seq_counter, s);
        snprintf(filename2, sizeof filename2, "Spezie_%d_Rabi_%d_%d.txt", 2, seq_counter, s);
        Output_rabi_freq_list(filename, filename2, seq.Nk);
      }
      if (seq.no_of_chirps > 1 && nrm > 0) {
        compute_rabi_integrals();
        list<double> tmp = m_rabi_freq_list.back();
        tmp.push_front(chirp_rate[0]);
        tmp.push_front(s);
        m_chirps_list.push_back(tmp);
      }
      // the scan restarts from the files of the sequence's start time; a file
      // that does not open leaves the fields as they are
      if (seq.no_of_chirps > 1 && s < seq.no_of_chirps - 1) {
        for (int k = 0; k < no_int_states; k++) {
          snprintf(filename, sizeof filename, "%.3f_%d.bin", backup_t, k + 1);
          this->reload(filename, k);
        }
        m_header.t = backup_t;
      }
    }
    if (seq.no_of_chirps > 1) {
      snprintf(filename, sizeof filename, "Chirp_%d.txt", seq_counter);
      Output_chirps_list(filename);
    }
    seq_counter++;
  }
  this->finish_output();
}

#endif
