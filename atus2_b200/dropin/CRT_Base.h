// CRT_Base.h (drop-in) -- real-time propagation of no_int_states coupled
// components in dim dimensions, with the interface of ATUS-2's
// template <class T, int dim, int no_int_states> class CRT_Base
// (include/CRT_Base.h:47-130), running on the GPU through libatus_gpu.so.
//
// The fields live in one GPU context; m_fields[c] is the GPU-backed field
// class T (cft_base.h) bound to component c, whose host mirror is what
// Getp2In() returns.  A program written for ATUS-2 compiles against these
// headers unchanged:
//   * run_sequence() follows CRT_Base::run_sequence (include/CRT_Base.h:
//     684-841): sequence loop, set_momentum, the Strang block
//     half, (V, full)^(Nk-1), V, half, file output and particle numbers;
//   * a sequence whose tag is in m_gpu_steps runs each block as one fused
//     GPU call (atus_strang_block); the tags are the step functions the
//     reference defines for this class ("freeprop" here; CRT_Base_IF and
//     CRT_Base_IF_2 add theirs), so a program's own registration under such
//     a tag is taken to be that same step.  ATUS_HOST_STEPS="tag,tag" makes
//     the listed tags run the program's registered function instead;
//   * any other tag in m_map_stepfcts runs as the program wrote it, on the
//     host mirror (download before, upload after, by the field classes),
//     with the kinetic steps on the GPU;
//   * m_Potential is uploaded when run_sequence starts and after each
//     Setup_Potential call; the header time m_header.t follows every GPU step.
// The reference's host tables m_full_step / m_half_step do not exist: the
// kinetic phases are per-axis FP64 factors on the GPU, rebuilt by Init()
// with m_alpha as the GPU context holds it.
#ifndef ATUS_DROPIN_CRT_BASE_H
#define ATUS_DROPIN_CRT_BASE_H

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "CRT_shared.h"
#include "cft_base.h"

using namespace std;

template <class T, int dim, int no_int_states>
class CRT_Base : public CRT_shared {
 public:
  CRT_Base(ParameterHandler *);
  virtual ~CRT_Base();

  double Get_Particle_Number(const int comp = 0);

  void run_sequence();

  void Setup_Momentum(CPoint<dim>, const int comp = 0);
  void Expval_Position(CPoint<dim> &, const int comp = 0);
  void Expval_Momentum(CPoint<dim> &, const int comp = 0);
  void Save(double *, std::string);
  void Save(fftw_complex *, std::string);
  void Save_Phi(std::string, const int comp = 0);
  void Append_Phi(std::string, const int comp = 0);
  void Dump_2(ofstream &);

  void Set_custom_fct(StepFunction &fct) { m_custom_fct = fct; }

  void Init_Potential();
  void Setup_Potential(const int, const int, const double);

 protected:
  static void Do_FT_Step_full_Wrapper(void *, sequence_item &);
  static void Do_FT_Step_half_Wrapper(void *, sequence_item &);
  static void Do_NL_Step_Wrapper(void *, sequence_item &);
  static void Do_NL_Step_Wrapper_one(void *, sequence_item &);

  void Do_FT_Step_full();
  void Do_FT_Step_half();
  void Do_NL_Step();

  ParameterHandler *m_params;
  CPoint<dim> m_alpha;

  void Init();
  void Allocate();
  void LoadFiles();

  bool m_potenial_initialized;

  virtual bool run_custom_sequence(const sequence_item &) = 0;

  std::array<double, no_int_states * no_int_states> m_gs;
  std::array<T *, no_int_states> m_fields;
  std::array<vector<double>, no_int_states> m_Potential;
  std::map<std::string, StepFunction> m_map_stepfcts;
  StepFunction m_custom_fct;

  // ---- asynchronous file output of run_sequence
  // The files of an output point (Save_Phi / Append_Phi of every component)
  // are written from a snapshot: the fields are copied into a device staging
  // buffer (microseconds, on the compute stream), and a writer thread per
  // component copies its field to the host and writes its file while the next
  // block runs.  One output point is in flight at a time; finish_output()
  // waits for it (before the next one, before any file is read back, before a
  // custom function runs, and when run_sequence ends).  ATUS_SYNC_OUTPUT=1
  // writes synchronously instead.
  std::vector<std::vector<double>> m_out_buf;
  std::vector<std::thread> m_writers;
  void finish_output() {
    for (auto &t : m_writers) t.join();
    m_writers.clear();
  }
  void output_point(const char *fmt, bool append, int seq_counter = 0) {
    char filename[1024];
    std::vector<std::string> names;
    for (int k = 0; k < no_int_states; k++) {
      if (append) snprintf(filename, sizeof filename, fmt, seq_counter, k + 1);
      else snprintf(filename, sizeof filename, fmt, this->Get_t(), k + 1);
      names.push_back(filename);
    }
    const char *sync = std::getenv("ATUS_SYNC_OUTPUT");
    if (sync && sync[0] == '1') {
      for (int k = 0; k < no_int_states; k++) append ? Append_Phi(names[k], k) : Save_Phi(names[k], k);
      return;
    }
    finish_output();
    m_out_buf.resize(no_int_states);
    gpu_before();
    atus_check(m_gpu, atus_snapshot(m_gpu), "snapshot");
    const generic_header h = m_header;
    const size_t n = 2 * (size_t)m_no_of_pts;
    for (int k = 0; k < no_int_states; k++) {
      std::vector<double> *buf = &m_out_buf[k];
      m_writers.emplace_back([this, k, h, n, buf, name = names[k], append]() {
        buf->resize(n);
        if (atus_snapshot_read(m_gpu, k, buf->data()) != ATUS_OK) {
          std::cerr << "GPU error reading an output snapshot" << std::endl;
          exit(EXIT_FAILURE);
        }
        std::ofstream f(name, append ? (std::ofstream::binary | std::ofstream::app) : std::ofstream::binary);
        if (f.fail()) {
          std::cout << "File " << name << " could not be opened. Failbit: " << f.rdstate() << std::endl;
          exit(EXIT_FAILURE);
        }
        f.write(reinterpret_cast<const char *>(&h), sizeof(generic_header));
        f.write(reinterpret_cast<const char *>(buf->data()), sizeof(double) * n);
      });
    }
  }

  // ---- GPU side
  atus_ctx *m_gpu = nullptr;
  // tags whose blocks run as one fused GPU call, with their step kind
  std::map<std::string, int> m_gpu_steps;
  bool m_pot_dirty = false;

  // before a GPU operation: upload what the host changed, pass the header time
  void gpu_before() {
    for (int c = 0; c < no_int_states; c++) m_fields[c]->push();
    if (m_pot_dirty) flush_potential();
    atus_check(m_gpu, atus_set_time(m_gpu, m_header.t), "set_time");
  }
  // after a GPU operation that changed the fields: the mirrors are stale
  void gpu_after(bool fields_changed = true) {
    if (fields_changed)
      for (int c = 0; c < no_int_states; c++) m_fields[c]->device_changed();
    atus_check(m_gpu, atus_get_time(m_gpu, &m_header.t), "get_time");
  }
  void flush_potential() {
    for (int c = 0; c < no_int_states; c++)
      atus_check(m_gpu, atus_set_potential(m_gpu, c, m_potenial_initialized ? m_Potential[c].data() : nullptr),
                 "set_potential");
    m_pot_dirty = false;
  }
  // GPU step kind of a tag, or -1 when the registered host function runs
  int gpu_kind(const std::string &tag) const {
    auto it = m_gpu_steps.find(tag);
    if (it == m_gpu_steps.end()) return -1;
    if (const char *h = std::getenv("ATUS_HOST_STEPS")) {
      std::stringstream ss(h);
      std::string t;
      while (std::getline(ss, t, ','))
        if (t == tag && m_map_stepfcts.count(tag)) return -1;
    }
    return it->second;
  }
  // AMP_T of every potential step of the coming block (1 here; CRT_Base_IF
  // evaluates the envelope)
  virtual void pulse_amplitudes(const sequence_item &, int nk, std::vector<double> &F) { F.assign(nk, 1.0); }
  // laser and pulse-window parameters of the step (CRT_Base_IF uploads them)
  virtual void upload_step_parameters(const sequence_item &) {}

  // One block: half, (V, full)^(Nk-1), V, half (include/CRT_Base.h:776-786).
  void strang_block(sequence_item &seq, int Nk, StepFunction step_fct, StepFunction half_fct,
                    StepFunction full_fct) {
    const int kind = gpu_kind(seq.name);
    if (kind >= 0 && half_fct == &Do_FT_Step_half_Wrapper && full_fct == &Do_FT_Step_full_Wrapper) {
      upload_step_parameters(seq);
      std::vector<double> F;
      pulse_amplitudes(seq, Nk, F);
      gpu_before();
      atus_check(m_gpu, atus_strang_block(m_gpu, Nk, kind, F.data()), "strang_block");
      gpu_after();
      return;
    }
    (*half_fct)(this, seq);
    for (int j = 2; j <= Nk; j++) {
      (*step_fct)(this, seq);
      (*full_fct)(this, seq);
    }
    (*step_fct)(this, seq);
    (*half_fct)(this, seq);
  }
  // strang_block that also returns the Rabi sums of the block's final state
  // (component comps[c] with centres k0[c], all lists of one length) when the
  // block runs fused on the GPU: the sums are then taken inside its last
  // kinetic pass.  Returns false (sums untouched) when the block ran
  // otherwise; the caller computes them separately then.
  bool strang_block_rabi(sequence_item &seq, int Nk, StepFunction step_fct, StepFunction half_fct,
                         StepFunction full_fct, const std::vector<int> &comps,
                         const std::vector<const std::vector<CPoint<dim>> *> &k0, double thr,
                         std::vector<std::vector<double>> &sums) {
    const int kind = gpu_kind(seq.name);
    const size_t n = k0.empty() ? 0 : k0[0]->size();
    bool ok = kind >= 0 && half_fct == &Do_FT_Step_half_Wrapper && full_fct == &Do_FT_Step_full_Wrapper && n > 0 &&
              comps.size() * n <= 8;
    for (auto *l : k0) ok = ok && l->size() == n;
    if (!ok) {
      strang_block(seq, Nk, step_fct, half_fct, full_fct);
      return false;
    }
    upload_step_parameters(seq);
    std::vector<double> F, kk, out(comps.size() * n);
    pulse_amplitudes(seq, Nk, F);
    for (auto *l : k0)
      for (auto &p : *l)
        for (int a = 0; a < dim; a++) kk.push_back(p[a]);
    gpu_before();
    atus_check(m_gpu,
               atus_strang_block_rabi(m_gpu, Nk, kind, F.data(), (int)comps.size(), comps.data(), kk.data(), (int)n,
                                      thr, out.data()),
               "strang_block_rabi");
    gpu_after();
    sums.assign(comps.size(), std::vector<double>(n));
    for (size_t c = 0; c < comps.size(); c++)
      for (size_t m = 0; m < n; m++) sums[c][m] = out[c * n + m];
    return true;
  }
  // the registered step of a tag; as in the reference a tag nobody
  // registered ends the program (a GPU kind only speeds up a registered tag)
  StepFunction step_function(const std::string &tag) {
    auto it = m_map_stepfcts.find(tag);
    if (it != m_map_stepfcts.end()) return it->second;
    std::cerr << "Critical Error: Invalid squence name " << tag << "\n";
    exit(EXIT_FAILURE);
  }
  // set_momentum sequence item (include/CRT_Base.h:720-734)
  void set_momentum(const sequence_item &seq) {
    std::vector<double> v;
    std::stringstream ss(seq.content);
    std::string part;
    while (std::getline(ss, part, ',')) v.push_back(std::stod(part));
    CPoint<dim> P;
    for (int i = 0; i < dim && i < (int)v.size(); i++) P[i] = v[i];
    this->Setup_Momentum(P, seq.comp);
    std::cout << "FYI: started new sequence " << seq.name << "\n";
    std::cout << "FYI: momentum set for component " << seq.comp << "\n";
  }
  // reads component k of a .bin file into its mirror (a restart point)
  void reload(const std::string &filename, int k) {
    finish_output();
    std::ifstream f(filename, std::ifstream::binary);
    if (!f.is_open()) return;
    f.seekg(sizeof(generic_header), std::ifstream::beg);
    fftw_complex *p = m_fields[k]->Getp2In();
    f.read(reinterpret_cast<char *>(p), sizeof(fftw_complex) * m_no_of_pts);
    m_fields[k]->host_changed();
  }
  void print_sequence(const sequence_item &seq, int seq_counter, double max_duration, int Na, int Nk) {
    std::cout << "FYI: started new sequence " << seq.name << "\n";
    std::cout << "FYI: sequence no : " << seq_counter << "\n";
    std::cout << "FYI: duration    : " << max_duration << "\n";
    std::cout << "FYI: dt          : " << seq.dt << "\n";
    std::cout << "FYI: Na          : " << Na << "\n";
    std::cout << "FYI: Nk          : " << Nk << "\n";
    std::cout << "FYI: Na*Nk*dt    : " << double(Na * Nk) * seq.dt << "\n";
  }
};

// Constructor (include/CRT_Base.h:138-175): header of FILENAME, fields and
// their files, the kinetic phases (Init) -- before Alpha_1 is read, as in the
// reference, so the phases hold alpha = 0 until the first Set_dt -- the step
// tags, g_ij and alpha, and dt of the ALGORITHM section.
template <class T, int dim, int no_int_states>
CRT_Base<T, dim, no_int_states>::CRT_Base(ParameterHandler *params) {
  m_params = params;
  Read_header(params->Get_simulation("FILENAME"), dim);
  if (m_header.nDims != dim) throw std::string("header.nDims does not match the program dimension");
  const atus_grid g = abi_grid(dim);
  atus_check(nullptr, atus_create(&g, no_int_states, atus_precision_from_env(), &m_gpu), "atus_create");
  Allocate();
  LoadFiles();
  Init();

  m_map_stepfcts["half_step"] = &Do_FT_Step_half_Wrapper;
  m_map_stepfcts["full_step"] = &Do_FT_Step_full_Wrapper;
  m_map_stepfcts["freeprop"] = &Do_NL_Step_Wrapper;
  m_map_stepfcts["freeprop_lin"] = &Do_NL_Step_Wrapper_one;
  m_gpu_steps["freeprop"] = ATUS_STEP_NL;
  m_custom_fct = nullptr;
  m_potenial_initialized = false;

  for (int i = 0; i < no_int_states; i++)
    for (int j = 0; j < no_int_states; j++)
      m_gs[j + no_int_states * i] = m_params->Get_VConstant("GS_" + std::to_string(i + 1), j);
  atus_check(m_gpu, atus_set_gs(m_gpu, m_gs.data()), "set_gs");
  for (int i = 0; i < dim; i++) m_alpha[i] = m_params->Get_VConstant("Alpha_1", i);
  double a[3] = {0, 0, 0};
  for (int i = 0; i < dim; i++) a[i] = m_alpha[i];
  for (int c = 0; c < no_int_states; c++) atus_check(m_gpu, atus_set_alpha(m_gpu, c, a), "set_alpha");
  m_header.dt = params->Get_dt();
}

template <class T, int dim, int no_int_states>
CRT_Base<T, dim, no_int_states>::~CRT_Base() {
  finish_output();
  for (int i = 0; i < no_int_states; i++) delete m_fields[i];
  atus_destroy(m_gpu);
}

template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Allocate() {
  for (int i = 0; i < no_int_states; i++) {
    m_fields[i] = new T(m_header);
    m_fields[i]->SetFix(false);
    m_fields[i]->atus_bind(m_gpu, i);
  }
}

// LoadFiles (include/CRT_Base.h:206-240): FILENAME, FILENAME_2, ...
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::LoadFiles() {
  for (int i = 0; i < no_int_states; i++) {
    const std::string key = (i == 0) ? "FILENAME" : "FILENAME_" + std::to_string(i + 1);
    std::ifstream in(m_params->Get_simulation(key), std::ifstream::binary);
    if (!in.is_open()) throw std::string("Could not open file " + m_params->Get_simulation(key) + "\n");
    in.seekg(sizeof(generic_header), std::ifstream::beg);
    in.read(reinterpret_cast<char *>(m_fields[i]->Getp2In()), sizeof(fftw_complex) * m_no_of_pts);
  }
}

// Init (include/CRT_Base.h:252-274): kinetic phases for m_header.dt with the
// context's alpha.
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Init() {
  atus_check(m_gpu, atus_set_dt(m_gpu, m_header.dt), "set_dt");
}

template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Init_Potential() {
  for (auto &v : m_Potential) v.resize(m_no_of_pts, 0);
  m_potenial_initialized = true;
  m_pot_dirty = true;
}

template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Setup_Potential(const int comp, const int index, const double val) {
  if (!m_potenial_initialized) {
    std::cerr << "Potential not initialized. You forgot to invoke Init_Potential." << std::endl;
    throw std::string("Potential not initialized");
  }
  assert(comp > -1 && comp < no_int_states);
  assert(index > -1 && index < m_no_of_pts);
  m_Potential[comp][index] = val;
  m_pot_dirty = true;
}

template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Do_FT_Step_full_Wrapper(void *ptr, sequence_item &) {
  static_cast<CRT_Base *>(ptr)->Do_FT_Step_full();
}
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Do_FT_Step_half_Wrapper(void *ptr, sequence_item &) {
  static_cast<CRT_Base *>(ptr)->Do_FT_Step_half();
}
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Do_NL_Step_Wrapper(void *ptr, sequence_item &) {
  static_cast<CRT_Base *>(ptr)->Do_NL_Step();
}
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Do_NL_Step_Wrapper_one(void *, sequence_item &) {}

// Do_FT_Step_full / _half (include/CRT_Base.h:336-392): FFT, phase, IFFT of
// every component, t += dt or dt/2
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Do_FT_Step_full() {
  gpu_before();
  atus_check(m_gpu, atus_ft_step(m_gpu, 0), "ft_step");
  gpu_after();
}
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Do_FT_Step_half() {
  gpu_before();
  atus_check(m_gpu, atus_ft_step(m_gpu, 1), "ft_step");
  gpu_after();
}

// Do_NL_Step (include/CRT_Base.h:396-441): exp(-i dt (V_i + sum_j g_ij |psi_j|^2))
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Do_NL_Step() {
  gpu_before();
  atus_check(m_gpu, atus_nl_step(m_gpu, ATUS_STEP_NL, 1.0), "nl_step");
  gpu_after();
}

template <class T, int dim, int no_int_states>
double CRT_Base<T, dim, no_int_states>::Get_Particle_Number(const int comp) {
  if (comp < 0 || comp > no_int_states) throw std::string("Error in Get_Particle_Number: comp out of bounds\n");
  gpu_before();
  double n = 0;
  atus_check(m_gpu, atus_particle_number(m_gpu, comp, &n), "particle_number");
  gpu_after(false);
  return n;
}

// Setup_Momentum (include/CRT_Base.h:448-473): psi *= exp(i p.x)
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Setup_Momentum(CPoint<dim> p, const int comp) {
  if (comp < 0 || comp > no_int_states) throw std::string("Error in Setup_Momentum: comp out of bounds\n");
  gpu_before();
  atus_check(m_gpu, atus_setup_momentum(m_gpu, comp, p.data()), "setup_momentum");
  gpu_after();
}

template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Expval_Position(CPoint<dim> &r, const int comp) {
  gpu_before();
  atus_check(m_gpu, atus_expval_position(m_gpu, comp, r.data()), "expval_position");
  gpu_after(false);
}
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Expval_Momentum(CPoint<dim> &r, const int comp) {
  gpu_before();
  atus_check(m_gpu, atus_expval_momentum(m_gpu, comp, r.data()), "expval_momentum");
  gpu_after(false);
}

// Save (include/CRT_Base.h:649-678): header and N values; a real array is
// written with bComplex = 0 and N doubles
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Save(double *data, std::string filename) {
  generic_header h = m_header;
  h.bComplex = false;
  std::ofstream f(filename, std::ofstream::binary);
  f.write(reinterpret_cast<const char *>(&h), sizeof(generic_header));
  f.write(reinterpret_cast<const char *>(data), sizeof(double) * m_no_of_pts);
}
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Save(fftw_complex *data, std::string filename) {
  std::ofstream f(filename, std::ofstream::binary);
  f.write(reinterpret_cast<const char *>(&m_header), sizeof(generic_header));
  f.write(reinterpret_cast<const char *>(data), sizeof(fftw_complex) * m_no_of_pts);
}

// Save_Phi / Append_Phi (include/CRT_Base.h:606-641)
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Save_Phi(std::string filename, const int comp) {
  finish_output();
  std::ofstream f(filename, std::ofstream::binary);
  f.write(reinterpret_cast<const char *>(&m_header), sizeof(generic_header));
  f.write(reinterpret_cast<const char *>(m_fields[comp]->host_view()), sizeof(fftw_complex) * m_no_of_pts);
}
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Append_Phi(std::string filename, const int comp) {
  finish_output();
  std::ofstream f(filename, std::ofstream::binary | std::ofstream::app);
  if (f.fail()) {
    std::cout << "File " << filename << " could not be opened. Failbit: " << f.rdstate() << std::endl;
    exit(EXIT_FAILURE);
  }
  f.write(reinterpret_cast<const char *>(&m_header), sizeof(generic_header));
  f.write(reinterpret_cast<const char *>(m_fields[comp]->host_view()), sizeof(fftw_complex) * m_no_of_pts);
}

template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::Dump_2(ofstream &stream) {
  stream << m_header.t << "\t";
}

template <class T, int dim, int no_int_states>
ofstream &operator<<(ofstream &stream, CRT_Base<T, dim, no_int_states> &obj) {
  obj.Dump_2(stream);
  return stream;
}

// run_sequence (include/CRT_Base.h:684-841)
template <class T, int dim, int no_int_states>
void CRT_Base<T, dim, no_int_states>::run_sequence() {
  char filename[1024];
  std::cout << "FYI: Found " << m_params->m_sequence.size() << " sequences." << std::endl;
  StepFunction half_fct = nullptr, full_fct = nullptr;
  try {
    half_fct = m_map_stepfcts.at("half_step");
    full_fct = m_map_stepfcts.at("full_step");
  } catch (const std::out_of_range &oor) {
    std::cerr << "Critical Error: Invalid fct ptr to ft_half_step or ft_full_step ()" << oor.what() << ")\n";
    exit(EXIT_FAILURE);
  }
  m_pot_dirty = true;  // the program may have filled m_Potential directly
  int seq_counter = 1;
  for (auto seq : m_params->m_sequence) {
    if (run_custom_sequence(seq)) continue;
    if (seq.name == "set_momentum") {
      set_momentum(seq);
      continue;
    }
    double max_duration = 0;
    for (double d : seq.duration)
      if (d > max_duration) max_duration = d;
    const int subN = int(max_duration / seq.dt);
    const int Nk = seq.Nk;
    const int Na = subN / seq.Nk;
    print_sequence(seq, seq_counter, max_duration, Na, Nk);
    if (double(Na * Nk) * seq.dt != max_duration) std::cout << "FYI: double(Na*Nk)*seq.dt != max_duration\n";
    if (this->Get_dt() != seq.dt) this->Set_dt(seq.dt);
    StepFunction step_fct = step_function(seq.name);
    finish_output();
    for (int k = 0; k < no_int_states; k++) {
      snprintf(filename, sizeof filename, "Seq_%d_%d.bin", seq_counter, k + 1);
      std::remove(filename);
    }
    for (int i = 1; i <= Na; i++) {
      strang_block(seq, Nk, step_fct, half_fct, full_fct);
      std::cout << "t = " << std::to_string(m_header.t) << std::endl;
      if (seq.output_freq == freq::each) output_point("%.3f_%d.bin", false);
      if (seq.output_freq == freq::packed) output_point("Seq_%d_%d.bin", true, seq_counter);
      if (seq.compute_pn_freq == freq::each)
        for (int c = 0; c < no_int_states; c++)
          std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
      if (seq.custom_freq == freq::each && m_custom_fct != nullptr) {
        finish_output();
        (*m_custom_fct)(this, seq);
      }
    }
    if (seq.output_freq == freq::last) output_point("%.3f_%d.bin", false);
    if (seq.compute_pn_freq == freq::last)
      for (int c = 0; c < no_int_states; c++)
        std::cout << "N[" << c << "] = " << this->Get_Particle_Number(c) << std::endl;
    if (seq.custom_freq == freq::last && m_custom_fct != nullptr) {
      finish_output();
      (*m_custom_fct)(this, seq);
    }
    seq_counter++;
  }
  finish_output();
}

#endif
