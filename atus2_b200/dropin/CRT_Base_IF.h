// CRT_Base_IF.h (drop-in) -- atom interferometry on top of CRT_Base, with
// the interface of ATUS-2's template <class T, int dim, int no_int_states>
// class CRT_Base_IF (include/CRT_Base_IF.h:49-117): laser members (beta,
// DeltaL, Amp, laser_k, laser_dk, laser_domh, phase, chirp_rate, chirp), the
// AMP_T envelope, Rabi momentum lists and their output, the chirp / phase
// scan of run_sequence, and the step functions freeprop (Do_NL_Step),
// bragg (Numerical_Bragg) and raman (Numerical_Raman).
//
// GPU step tags (fused blocks): "freeprop" (g|psi|^2 + beta x - DeltaL),
// "bragg", "raman", and "bragg_ad" -- the analytic two-level step of the
// bragg program (source/interferometry/src/bragg.cpp:185-304) for two
// components, the three-level step of double_bragg
// (source/interferometry/src/double_bragg.cpp:100-258) for three.  A program
// that registers "bragg_ad" (both programs do) gets these kernels for it.
#ifndef ATUS_DROPIN_CRT_BASE_IF_H
#define ATUS_DROPIN_CRT_BASE_IF_H

#include <cmath>
#include <cstring>
#include <list>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "CRT_Base.h"
#include "muParser.h"

using namespace std;

template <class T, int dim, int no_int_states>
class CRT_Base_IF : public CRT_Base<T, dim, no_int_states> {
 public:
  CRT_Base_IF(ParameterHandler *);
  virtual ~CRT_Base_IF() {}

  void run_sequence();

 protected:
  using CRT_Base<T, dim, no_int_states>::m_header;
  using CRT_Base<T, dim, no_int_states>::m_params;
  using CRT_Base<T, dim, no_int_states>::m_fields;
  using CRT_Base<T, dim, no_int_states>::m_custom_fct;
  using CRT_shared::m_no_of_pts;

  CPoint<dim> beta;
  std::array<double, no_int_states> DeltaL;
  std::array<double, 2> Amp, laser_k, laser_dk, laser_domh, phase, chirp_rate;
  double chirp;
  bool amp_is_t;

  static void Do_NL_Step_Wrapper(void *, sequence_item &);
  static void Numerical_Bragg_Wrapper(void *, sequence_item &);
  static void Numerical_Raman_Wrapper(void *, sequence_item &);

  void Do_NL_Step();
  void Numerical_Bragg();
  void Numerical_Raman();

  void UpdateParams();
  void Output_rabi_freq_list(string, const long long);
  void Output_chirps_list(string);

  virtual bool run_custom_sequence(const sequence_item &) = 0;

  double m_rabi_threshold;
  vector<CPoint<dim>> m_rabi_momentum_list;
  list<list<double>> m_rabi_freq_list;
  list<list<double>> m_chirps_list;

  void compute_rabi_integrals();

  double Amplitude_at_time();

  // ---- GPU side
  void upload_step_parameters(const sequence_item &) override { upload_laser(); }
  void upload_laser() {
    const atus_laser L = make_laser();
    atus_check(this->m_gpu, atus_set_laser(this->m_gpu, &L), "set_laser");
  }
  atus_laser make_laser() const {
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
    return L;
  }
  // AMP_T at t + dt/2 of every potential step of the coming block, with the
  // header-time additions of the block (include/CRT_Base_IF.h:170-198)
  void pulse_amplitudes(const sequence_item &, int nk, std::vector<double> &F) override {
    F.assign(nk, 1.0);
    if (!amp_is_t) return;
    const double dt = this->Get_dt();
    double time = 0;
    mu::Parser p;
    m_params->Setup_muParser(p);
    p.SetExpr(m_params->Get_simulation("AMP_T"));
    p.DefineVar("t", &time);
    double t = m_header.t + 0.5 * dt;  // after the leading half step
    for (int j = 0; j < nk; j++) {
      time = t + 0.5 * dt;
      F[j] = p.Eval();
      t += dt;
    }
  }
  // ---- phase scans side by side
  // One scan s >= 1 of a phase scan (chirp_mode 1) on its own clone of the
  // sequence's start state: Na fused blocks with the scan's laser, the
  // per-block and per-scan observables of run_sequence, its Rabi file; the
  // console lines go to `text` (printed in scan order by the caller) and the
  // scan's entry of the chirp list to `entry`.
  struct ScanJob {
    atus_ctx *ctx = nullptr;
    atus_laser laser{};
    int s = 0, kind = 0, Na = 0, Nk = 0, seq_counter = 0;
    const std::vector<std::vector<double>> *F = nullptr;
    std::vector<double> k0;
    int nrm = 0;
    double thr = 0, dt = 0, phase = 0;
    int rabi_freq = 0, pn_freq = 0;
    std::string rabi_header;
    std::string text;
    list<double> entry;
    int err = 0;
    std::string errmsg;
  };
  static void run_scan(ScanJob *j) {
    std::ostringstream out;
    list<list<double>> rabi;
    auto fail = [&](int r) {
      j->err = r;
      j->errmsg = atus_last_error(j->ctx);
    };
    auto sums = [&](std::vector<double> &v) {
      v.assign(j->nrm, 0.0);
      const int r = atus_rabi_integrals(j->ctx, j->k0.data(), j->nrm, j->thr, v.data());
      if (r != ATUS_OK) fail(r);
    };
    int r = atus_set_laser(j->ctx, &j->laser);
    if (r != ATUS_OK) return fail(r);
    for (int i = 0; i < j->Na && !j->err; i++) {
      const double *F = (*j->F)[i].data();
      if (j->rabi_freq == freq::each && j->nrm > 0) {
        std::vector<double> v(j->nrm);
        const int c0 = 0;
        r = atus_strang_block_rabi(j->ctx, j->Nk, j->kind, F, 1, &c0, j->k0.data(), j->nrm, j->thr, v.data());
        if (r != ATUS_OK) return fail(r);
        rabi.push_back(list<double>(v.begin(), v.end()));
      } else {
        r = atus_strang_block(j->ctx, j->Nk, j->kind, F);
        if (r != ATUS_OK) return fail(r);
      }
      double t = 0;
      atus_get_time(j->ctx, &t);
      out << "t = " << to_string(t) << std::endl;
      if (j->pn_freq == freq::each)
        for (int c = 0; c < no_int_states; c++) {
          double n = 0;
          atus_particle_number(j->ctx, c, &n);
          out << "N[" << c << "] = " << n << std::endl;
        }
      if (j->rabi_freq == freq::each && j->nrm == 0)
        std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << endl;
    }
    if (j->err) return;
    double t_end = 0;
    atus_get_time(j->ctx, &t_end);
    if (j->pn_freq == freq::last)
      for (int c = 0; c < no_int_states; c++) {
        double n = 0;
        atus_particle_number(j->ctx, c, &n);
        out << "N[" << c << "] = " << n << std::endl;
      }
    if (j->rabi_freq == freq::last && j->nrm > 0) {
      std::vector<double> v;
      sums(v);
      rabi.push_back(list<double>(v.begin(), v.end()));
      out << "Rabi output for timestep ";
      for (auto &row : rabi) {
        out << t_end << "\n";
        for (double x : row) out << x << "\t";
        out << endl;
      }
    }
    if (j->rabi_freq == freq::each) {
      char filename[1024];
      snprintf(filename, sizeof filename, "Rabi_%d_%d.txt", j->seq_counter, j->s);
      ofstream txt(filename);
      double t = 0;
      txt << j->rabi_header << endl;
      for (auto &row : rabi) {
        txt << t << "\t";
        for (double x : row) txt << x << "\t";
        txt << endl;
        t += j->dt * double(j->Nk);
      }
    }
    if (j->nrm > 0) {
      std::vector<double> v;
      sums(v);
      j->entry = list<double>(v.begin(), v.end());
      j->entry.push_front(j->phase);
      j->entry.push_front(j->s);
    }
    j->text = out.str();
  }

  // one potential step of GPU kind `kind` at the current header time
  void gpu_potential_step(int kind) {
    upload_laser();
    const double F = Amplitude_at_time();
    this->gpu_before();
    atus_check(this->m_gpu, atus_nl_step(this->m_gpu, kind, F), "nl_step");
    this->gpu_after();
  }
};

// Constructor (include/CRT_Base_IF.h:124-129)
template <class T, int dim, int no_int_states>
CRT_Base_IF<T, dim, no_int_states>::CRT_Base_IF(ParameterHandler *params)
    : CRT_Base<T, dim, no_int_states>(params), chirp(0), amp_is_t(false), m_rabi_threshold(0) {
  DeltaL.fill(0);
  Amp.fill(0);
  laser_k.fill(0);
  laser_dk.fill(0);
  laser_domh.fill(0);
  phase.fill(0);
  chirp_rate.fill(0);
  this->m_map_stepfcts["freeprop"] = &Do_NL_Step_Wrapper;
  this->m_map_stepfcts["bragg"] = &Numerical_Bragg_Wrapper;
  this->m_map_stepfcts["raman"] = &Numerical_Raman_Wrapper;
  this->m_gpu_steps["freeprop"] = ATUS_STEP_NL_IF;
  this->m_gpu_steps["bragg"] = ATUS_STEP_NUMERICAL_BRAGG;
  this->m_gpu_steps["raman"] = ATUS_STEP_NUMERICAL_RAMAN;
  if (no_int_states == 2) this->m_gpu_steps["bragg_ad"] = ATUS_STEP_BRAGG_AD;
  if (no_int_states == 3) this->m_gpu_steps["bragg_ad"] = ATUS_STEP_DOUBLE_BRAGG_AD;
  UpdateParams();
}

// UpdateParams (include/CRT_Base_IF.h:144-168)
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::UpdateParams() {
  for (int i = 0; i < dim; i++) beta[i] = m_params->Get_VConstant("Beta", i);
  for (int i = 0; i < no_int_states; i++) DeltaL[i] = m_params->Get_VConstant("Delta_L", i);
  try {
    Amp[0] = m_params->Get_VConstant("Amp_1", 0);
    Amp[1] = m_params->Get_VConstant("Amp_1", 1);
    laser_k[0] = m_params->Get_Constant("laser_k");
    laser_dk[0] = m_params->Get_Constant("laser_dk");
    laser_domh[0] = m_params->Get_Constant("laser_domh");
    m_rabi_threshold = m_params->Get_Constant("rabi_threshold");
    chirp = m_params->Get_Constant("chirp");
  } catch (std::string &str) {
    cout << str << endl;
    exit(EXIT_FAILURE);
  }
}

// Amplitude_at_time (include/CRT_Base_IF.h:170-198): AMP_T(t + dt/2), else 1
template <class T, int dim, int no_int_states>
double CRT_Base_IF<T, dim, no_int_states>::Amplitude_at_time() {
  if (!amp_is_t) return 1;
  double time;
  try {
    mu::Parser p;
    m_params->Setup_muParser(p);
    p.SetExpr(m_params->Get_simulation("AMP_T"));
    p.DefineVar("t", &time);
    time = this->Get_t() + 0.5 * this->Get_dt();
    return p.Eval();
  } catch (mu::Parser::exception_type &e) {
    cout << "Message:  " << e.GetMsg() << "\n";
    cout << "Formula:  " << e.GetExpr() << "\n";
    cout << "Token:    " << e.GetToken() << "\n";
    cout << "Position: " << e.GetPos() << "\n";
    cout << "Errc:     " << e.GetCode() << "\n";
    exit(EXIT_FAILURE);
  }
}

// compute_rabi_integrals (include/CRT_Base_IF.h:207-281): m_ar_k sum |psi_0^(k)|^2
// over the balls |k - k0| < m_rabi_threshold, on the GPU
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::compute_rabi_integrals() {
  const int n = (int)m_rabi_momentum_list.size();
  if (n == 0) {
    std::cerr << "WARNING: Rabi momentum list is empty. Cannot compute rabi frquencies." << endl;
    return;
  }
  std::vector<double> k0, res(n);
  for (auto &p : m_rabi_momentum_list)
    for (int a = 0; a < dim; a++) k0.push_back(p[a]);
  this->gpu_before();
  atus_check(this->m_gpu, atus_rabi_integrals(this->m_gpu, k0.data(), n, m_rabi_threshold, res.data()), "rabi");
  this->gpu_after(false);
  m_rabi_freq_list.push_back(list<double>(res.begin(), res.end()));
}

template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Output_rabi_freq_list(string filename, const long long Nk) {
  ofstream txt(filename);
  double t = 0;
  txt << "# time \t";
  for (auto &p : m_rabi_momentum_list) txt << p << "\t";
  txt << endl;
  for (auto &row : m_rabi_freq_list) {
    txt << t << "\t";
    for (double v : row) txt << v << "\t";
    txt << endl;
    t += m_header.dt * double(Nk);
  }
}

template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Output_chirps_list(string filename) {
  ofstream txt(filename);
  txt << "# Step \t Chirp \t ";
  for (auto &p : m_rabi_momentum_list) txt << p << "\t";
  txt << endl;
  for (auto &row : m_chirps_list) {
    for (double v : row) {
      txt.precision(8);
      txt << v << "\t";
    }
    txt << endl;
  }
}

template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Do_NL_Step_Wrapper(void *ptr, sequence_item &) {
  static_cast<CRT_Base_IF *>(ptr)->Do_NL_Step();
}
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Numerical_Bragg_Wrapper(void *ptr, sequence_item &) {
  static_cast<CRT_Base_IF *>(ptr)->Numerical_Bragg();
}
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Numerical_Raman_Wrapper(void *ptr, sequence_item &) {
  static_cast<CRT_Base_IF *>(ptr)->Numerical_Raman();
}

// Do_NL_Step (include/CRT_Base_IF.h:380-419), Numerical_Bragg / Numerical_Raman
// (include/CRT_Base_IF.h:426-632): one potential step on the GPU
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Do_NL_Step() {
  gpu_potential_step(ATUS_STEP_NL_IF);
}
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Numerical_Bragg() {
  gpu_potential_step(ATUS_STEP_NUMERICAL_BRAGG);
}
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::Numerical_Raman() {
  gpu_potential_step(ATUS_STEP_NUMERICAL_RAMAN);
}

// run_sequence (include/CRT_Base_IF.h:638-946)
template <class T, int dim, int no_int_states>
void CRT_Base_IF<T, dim, no_int_states>::run_sequence() {
  char filename[1024];
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
    this->print_sequence(seq, seq_counter, max_duration, Na, Nk);
    if (m_params->Has_simulation("AMP_T")) {
      std::cout << "FYI: Amp is      : " << m_params->Get_simulation("AMP_T") << "\n";
      amp_is_t = true;
    } else {
      std::cout << "FYI: Amp is      : 1" << std::endl;
      amp_is_t = false;
    }
    if (double(Na * Nk) * seq.dt != max_duration) std::cout << "FYI: double(Na*Nk)*seq.dt != max_duration\n";
    if (this->Get_dt() != seq.dt) this->Set_dt(seq.dt);
    StepFunction step_fct = this->step_function(seq.name);
    if (seq.name == "freeprop") seq.no_of_chirps = 1;
    const double backup_t = m_header.t;
    double backup_end_t = m_header.t;
    this->finish_output();
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
    // A phase scan (chirp_mode 1) has independent scans: each starts from this
    // state, with phase s 2 pi / n and chirp rates that do not depend on the
    // results (dw[s + 1] = (dw[s] + dw[s - 1]) / 2; the swap on dphi only
    // applies to the chirp scan).  Where the blocks run fused on the GPU and
    // no custom function touches the solver, scans 1..n-1 run side by side on
    // clones of the context while scan 0 runs here with all its outputs.
    const int gkind = this->gpu_kind(seq.name);
    const bool side = seq.no_of_chirps > 1 && seq.chirp_mode == 1 && gkind >= 0 &&
                      half_fct == &CRT_Base<T, dim, no_int_states>::Do_FT_Step_half_Wrapper &&
                      full_fct == &CRT_Base<T, dim, no_int_states>::Do_FT_Step_full_Wrapper &&
                      m_custom_fct == nullptr && !std::getenv("ATUS_SEQUENTIAL_SCANS");
    std::vector<ScanJob> jobs;
    std::vector<std::thread> workers;
    std::vector<std::vector<double>> Fs;
    if (side) {
      for (int s = 1; s + 1 < seq.no_of_chirps; s++) dw[s + 1] = (dw[s] + dw[s - 1]) / 2;
      // pulse amplitudes of every block, with the header-time additions of the blocks
      const double save_t = m_header.t, dt = this->Get_dt();
      double t = m_header.t;
      Fs.resize(Na);
      for (int i = 0; i < Na; i++) {
        m_header.t = t;
        this->pulse_amplitudes(seq, Nk, Fs[i]);
        t += 0.5 * dt;
        for (int j = 0; j < Nk; j++) t += (j == Nk - 1) ? 0.5 * dt : dt;
      }
      m_header.t = save_t;
      this->upload_step_parameters(seq);
      this->gpu_before();
      std::ostringstream hdr;
      hdr << "# time \t";
      for (auto &p : m_rabi_momentum_list) hdr << p << "\t";
      jobs.resize(seq.no_of_chirps - 1);
      for (int s = 1; s < seq.no_of_chirps; s++) {
        ScanJob &j = jobs[s - 1];
        atus_check(this->m_gpu, atus_clone(this->m_gpu, &j.ctx), "clone");
        j.laser = make_laser();
        j.phase = s * 2.0 * M_PI / (1.0 * seq.no_of_chirps);
        j.laser.phase[0] = j.phase;
        j.laser.chirp_rate[0] = dw[s];
        j.s = s;
        j.kind = gkind;
        j.Na = Na;
        j.Nk = Nk;
        j.seq_counter = seq_counter;
        j.F = &Fs;
        for (auto &p : m_rabi_momentum_list)
          for (int a = 0; a < dim; a++) j.k0.push_back(p[a]);
        j.nrm = nrm;
        j.thr = m_rabi_threshold;
        j.dt = m_header.dt;
        j.rabi_freq = seq.rabi_output_freq;
        j.pn_freq = seq.compute_pn_freq;
        j.rabi_header = hdr.str();
      }
      for (auto &j : jobs) workers.emplace_back(&CRT_Base_IF::run_scan, &j);
    }
    for (int s = 0; s < (side ? 1 : seq.no_of_chirps); ++s) {
      m_rabi_freq_list.clear();
      chirp_rate[0] = dw[s];
      if (seq.chirp_mode == 1) phase[0] = s * 2.0 * M_PI / (1.0 * seq.no_of_chirps);
      for (int i = 1; i <= Na; i++) {
        // with Rabi output each block, the sums come out of the block's last
        // kinetic pass where it runs fused on the GPU
        bool rabi_done = false;
        if (seq.rabi_output_freq == freq::each && nrm > 0) {
          std::vector<std::vector<double>> sums;
          rabi_done = this->strang_block_rabi(seq, Nk, step_fct, half_fct, full_fct, {0}, {&m_rabi_momentum_list},
                                              m_rabi_threshold, sums);
          if (rabi_done) m_rabi_freq_list.push_back(list<double>(sums[0].begin(), sums[0].end()));
        } else {
          this->strang_block(seq, Nk, step_fct, half_fct, full_fct);
        }
        std::cout << "t = " << to_string(m_header.t) << std::endl;
        if (seq.output_freq == freq::each && s == 0) this->output_point("%.3f_%d.bin", false);
        if (seq.output_freq == freq::packed && s == 0) this->output_point("Seq_%d_%d.bin", true, seq_counter);
        if (seq.compute_pn_freq == freq::each)
          for (int c = 0; c < no_int_states; c++)
            std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
        if (seq.rabi_output_freq == freq::each && !rabi_done) compute_rabi_integrals();
        if (seq.custom_freq == freq::each && m_custom_fct != nullptr) {
          this->finish_output();
          (*m_custom_fct)(this, seq);
        }
      }
      if (seq.output_freq == freq::last && s == 0) this->output_point("%.3f_%d.bin", false);
      if (seq.no_of_chirps > 1 && s == 0) {
        backup_end_t = this->Get_t();
        for (int k = 0; k < no_int_states; k++) {
          snprintf(filename, sizeof filename, "%.3f_%d.bin", this->Get_t(), k + 1);
          this->Save_Phi(filename, k);
        }
      }
      if (seq.compute_pn_freq == freq::last)
        for (int c = 0; c < no_int_states; c++)
          std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
      if (seq.custom_freq == freq::last && m_custom_fct != nullptr) {
        this->finish_output();
        (*m_custom_fct)(this, seq);
      }
      if (seq.rabi_output_freq == freq::last) {
        compute_rabi_integrals();
        cout << "Rabi output for timestep ";
        for (auto &row : m_rabi_freq_list) {
          cout << this->Get_t() << "\n";
          for (double v : row) cout << v << "\t";
          cout << endl;
        }
      }
      if (seq.rabi_output_freq == freq::each) {
        snprintf(filename, sizeof filename, "Rabi_%d_%d.txt", seq_counter, s);
        Output_rabi_freq_list(filename, seq.Nk);
      }
      if (seq.no_of_chirps > 1) {
        if (nrm > 0) {
          compute_rabi_integrals();
          list<double> tmp = m_rabi_freq_list.back();
          if (seq.chirp_mode == 1) {
            tmp.push_front(phase[0]);
          } else {
            dphi[s] = tmp.front();
            tmp.push_front(chirp_rate[0]);
          }
          tmp.push_front(s);
          m_chirps_list.push_back(tmp);
        }
        if (s < seq.no_of_chirps - 1 && !side) {
          for (int k = 0; k < no_int_states; k++) {
            snprintf(filename, sizeof filename, "%.3f_%d.bin", backup_t, k + 1);
            this->reload(filename, k);
          }
          m_header.t = backup_t;
        }
        if (s > 0 && s < seq.no_of_chirps - 1 && !side) {
          dw[s + 1] = (dw[s] + dw[s - 1]) / 2;
          if (dphi[s] - dphi[s - 1] < 0) {
            dw[s] = dw[s - 1];
            dphi[s] = dphi[s - 1];
          }
        }
      }
    }
    if (side) {  // the other scans, in scan order
      for (auto &w : workers) w.join();
      for (auto &j : jobs) {
        atus_destroy(j.ctx);
        if (j.err) {
          std::cerr << "GPU error in scan " << j.s << ": " << j.errmsg << " (code " << j.err << ")" << endl;
          exit(EXIT_FAILURE);
        }
        std::cout << j.text;
        if (nrm > 0) m_chirps_list.push_back(j.entry);
      }
    }
    if (seq.no_of_chirps > 1) {
      snprintf(filename, sizeof filename, "Chirp_%d.txt", seq_counter);
      Output_chirps_list(filename);
      for (int k = 0; k < no_int_states; k++) {
        snprintf(filename, sizeof filename, "%.3f_%d.bin", backup_end_t, k + 1);
        this->reload(filename, k);
      }
      m_header.t = backup_end_t;
    }
    seq_counter++;
  }
  this->finish_output();
}

#endif
