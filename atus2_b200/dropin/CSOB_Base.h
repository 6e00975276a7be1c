// CSOB_Base.h (drop-in) -- ground states by Sobolev-gradient descent, with
// the interface of ATUS-2's template <class T, int dim, int no_wf> class
// CSOB_Base (include/CSOB_Base.h:42-90), running on the GPU through
// libatus_gpu.so.
//
// The grid comes from the ALGORITHM section as in the reference constructor
// (include/CSOB_Base.h:96-190).  m_Psi and m_Potential are host arrays the
// program fills (sob_solver.cpp's Setup_Guess / Setup_Potential write them
// after construction); run() uploads them, runs the descent of
// CSOB_Base::run (include/CSOB_Base.h:426-505: renormalise, Sobolev
// gradient, projection, residual, update until m_res_tot <= m_epsilon) on
// the GPU with the reference's per-iteration console lines, and downloads the
// result into m_Psi.  The operator tables m_operator_fs and
// m_Laplace_operator_fs are filled on the host as Init() does in the
// reference (the GPU builds its own from alpha); m_Laplace_Psi and m_Psi_sob
// are host arrays kept for subclasses (the GPU keeps its own copies).
#ifndef ATUS_DROPIN_CSOB_BASE_H
#define ATUS_DROPIN_CSOB_BASE_H

#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "CRT_shared.h"
#include "cft_base.h"

using namespace std;

template <class T, int dim, int no_wf>
class CSOB_Base : public CRT_shared {
 public:
  CSOB_Base(ParameterHandler *);
  virtual ~CSOB_Base();

  double Get_Particle_Number(const int comp = 0);

  void run();

  void Save(double *, std::string);
  void Save(fftw_complex *, std::string);
  void Save(std::vector<std::string>, bool = false);
  void Save_Zero();
  void Dump_2(ofstream &stream) { stream << m_header.t << "\t"; }

 protected:
  double m_res_tot;
  double m_epsilon;
  double m_stepsize;

  void Init_Potential() {}
  void Compute_mu();
  void Renormalize_All_Psi();

  ParameterHandler *m_params;

  std::array<double, no_wf> m_mu;
  std::array<double, no_wf> m_N;
  std::array<CPoint<dim>, no_wf> m_alpha;
  std::array<double *, no_wf> m_operator_fs;
  std::array<double *, no_wf> m_Laplace_operator_fs;
  std::array<double *, no_wf> m_Potential;

  std::array<fftw_complex *, no_wf> m_Psi;
  std::array<fftw_complex *, no_wf> m_Laplace_Psi;
  std::array<fftw_complex *, no_wf> m_Psi_sob;

  std::array<double, dim> m_res;
  std::array<double, no_wf * no_wf> m_gs;
  std::array<T *, no_wf> m_fields;

  void Init();
  void Allocate();

  // ---- GPU side
  atus_ctx *m_gpu = nullptr;
  // m_Psi and m_Potential to the GPU, the descent's parameters with them
  void upload() {
    for (int i = 0; i < no_wf; i++) {
      atus_check(m_gpu, atus_upload_psi(m_gpu, i, &m_Psi[i][0][0]), "upload");
      atus_check(m_gpu, atus_set_potential(m_gpu, i, m_Potential[i]), "set_potential");
    }
    double a[4] = {0, 0, 0, 0};
    for (int i = 0; i < no_wf; i++) a[i] = m_alpha[i][0];
    atus_check(m_gpu, atus_sob_init(m_gpu, a, m_stepsize), "sob_init");
  }
  void download() {
    for (int i = 0; i < no_wf; i++) atus_check(m_gpu, atus_download_psi(m_gpu, i, &m_Psi[i][0][0]), "download");
  }
};

// Constructor (include/CSOB_Base.h:96-190)
template <class T, int dim, int no_wf>
CSOB_Base<T, dim, no_wf>::CSOB_Base(ParameterHandler *params) {
  m_params = params;
  m_header = {};
  m_header.nself = sizeof(generic_header);
  m_header.bAtom = 1;
  m_header.bComplex = 1;
  m_header.nDatatyp = sizeof(fftw_complex);
  m_header.nDims = dim;
  m_header.dt = 0.01;
  m_header.nDimX = params->Get_NX();
  m_header.nDimY = dim >= 2 ? params->Get_NY() : 1;
  m_header.nDimZ = dim >= 3 ? params->Get_NZ() : 1;
  m_header.xMax = params->Get_xMax();
  m_header.xMin = params->Get_xMin();
  m_header.dx = fabs(m_header.xMax - m_header.xMin) / double(m_header.nDimX);
  m_header.dkx = 2 * M_PI / fabs(m_header.xMax - m_header.xMin);
  if (dim >= 2) {
    m_header.yMax = params->Get_yMax();
    m_header.yMin = params->Get_yMin();
    m_header.dy = fabs(m_header.yMax - m_header.yMin) / double(m_header.nDimY);
    m_header.dky = 2 * M_PI / fabs(m_header.yMax - m_header.yMin);
  }
  if (dim >= 3) {
    m_header.zMax = params->Get_zMax();
    m_header.zMin = params->Get_zMin();
    m_header.dz = fabs(m_header.zMax - m_header.zMin) / double(m_header.nDimZ);
    m_header.dkz = 2 * M_PI / fabs(m_header.zMax - m_header.zMin);
  }
  set_geometry(dim);
  for (int i = 0; i < no_wf; i++)
    for (int j = 0; j < no_wf; j++)
      m_gs[j + no_wf * i] = m_params->Get_VConstant("GS_" + std::to_string(i + 1), j) *
                            sqrt(m_params->Get_VConstant("N", i)) * sqrt(m_params->Get_VConstant("N", j));
  for (int i = 0; i < no_wf; i++) m_alpha[i] = m_params->Get_VConstant("Alpha_" + std::to_string(i + 1), 0);
  m_header.dt = params->Get_dt();
  m_epsilon = m_params->Get_Constant("epsilon");
  m_stepsize = m_params->Get_Constant("stepsize");
  m_res_tot = 0;
  m_mu.fill(0);
  m_N.fill(0);
  m_res.fill(0);
  const atus_grid g = abi_grid(dim);
  atus_check(nullptr, atus_create(&g, no_wf, ATUS_PREC_FP64, &m_gpu), "atus_create");
  atus_check(m_gpu, atus_set_gs(m_gpu, m_gs.data()), "set_gs");
  Allocate();
  Init();
}

template <class T, int dim, int no_wf>
CSOB_Base<T, dim, no_wf>::~CSOB_Base() {
  for (int i = 0; i < no_wf; i++) {
    delete m_fields[i];
    fftw_free(m_operator_fs[i]);
    fftw_free(m_Laplace_operator_fs[i]);
    fftw_free(m_Potential[i]);
    fftw_free(m_Psi[i]);
    fftw_free(m_Laplace_Psi[i]);
    fftw_free(m_Psi_sob[i]);
  }
  atus_destroy(m_gpu);
}

template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Allocate() {
  for (int i = 0; i < no_wf; i++) {
    m_operator_fs[i] = fftw_alloc_real(m_no_of_pts);
    m_Laplace_operator_fs[i] = fftw_alloc_real(m_no_of_pts);
    m_Potential[i] = fftw_alloc_real(m_no_of_pts);
    m_Psi[i] = fftw_alloc_complex(m_no_of_pts);
    m_Laplace_Psi[i] = fftw_alloc_complex(m_no_of_pts);
    m_Psi_sob[i] = fftw_alloc_complex(m_no_of_pts);
    std::memset(m_Potential[i], 0, sizeof(double) * m_no_of_pts);
    std::memset(m_Psi[i], 0, sizeof(fftw_complex) * m_no_of_pts);
    m_fields[i] = new T(m_header);
    m_fields[i]->SetFix(false);
  }
}

// Init (include/CSOB_Base.h:228-248): 1/(1 + alpha k^2) and -alpha k^2
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Init() {
  for (int j = 0; j < no_wf; j++)
    for (int i = 0; i < m_no_of_pts; i++) {
      CPoint<dim> k = m_fields[0]->Get_k(i);
      const double phi = k.scale(m_alpha[j]) * k;
      m_operator_fs[j][i] = 1.0 / (1.0 + phi);
      m_Laplace_operator_fs[j][i] = -phi;
    }
}

// Get_Particle_Number (include/CSOB_Base.h:508-519): m_ar sum |m_Psi|^2
template <class T, int dim, int no_wf>
double CSOB_Base<T, dim, no_wf>::Get_Particle_Number(const int comp) {
  if (comp < 0 || comp > no_wf) throw std::string("Error in Get_Particle_Number: comp out of bounds\n");
  atus_check(m_gpu, atus_upload_psi(m_gpu, comp, &m_Psi[comp][0][0]), "upload");
  double n = 0;
  atus_check(m_gpu, atus_particle_number(m_gpu, comp, &n), "particle_number");
  return n;
}

// Renormalize_All_Psi (include/CSOB_Base.h:521-543), on the GPU copy
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Renormalize_All_Psi() {
  upload();
  atus_check(m_gpu, atus_sob_renormalize(m_gpu), "renormalize");
  download();
  m_N.fill(1);
}

// mu_i = m_ar sum[-Re(psi* Lap psi) + (V + sum_j g_ij |psi_j|^2) |psi_i|^2]
// (the formula of include/CSOB_Base.h:399-424) of m_Psi, into m_mu
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Compute_mu() {
  upload();
  double mu[4] = {0, 0, 0, 0};
  atus_check(m_gpu, atus_sob_mu(m_gpu, mu), "sob_mu");
  for (int i = 0; i < no_wf; i++) m_mu[i] = mu[i];
}

// run (include/CSOB_Base.h:426-505)
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::run() {
  upload();
  atus_check(m_gpu, atus_sob_renormalize(m_gpu), "renormalize");
  int counter = 0;
  do {
    double N[ATUS_MAX_COMP];
    atus_check(m_gpu, atus_sob_iterate(m_gpu, 1, &m_res_tot, N), "sob_iterate");
    bool brenorm = false;
    for (int i = 0; i < no_wf; i++) {
      m_N[i] = N[i];
      if (fabs(N[i] - 1) > 1e-5) brenorm = true;
      cout << "N[" << i << "] = " << N[i] << endl;
    }
    printf("brenorm = %s\n", brenorm ? "true" : "false");
    cout << "--- " << counter << endl;
    cout << "res " << m_res_tot << endl;
    counter++;
  } while (m_res_tot > m_epsilon);
  download();
}

// Save (include/CSOB_Base.h:545-590)
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Save(double *data, std::string filename) {
  generic_header h = m_header;
  h.bComplex = false;
  h.nDatatyp = sizeof(double);
  ofstream f(filename, ofstream::binary);
  f.write(reinterpret_cast<const char *>(&h), sizeof(generic_header));
  f.write(reinterpret_cast<const char *>(data), sizeof(double) * m_no_of_pts);
}
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Save(fftw_complex *data, std::string filename) {
  cout << filename << endl;
  ofstream f(filename, ofstream::binary);
  f.write(reinterpret_cast<const char *>(&m_header), sizeof(generic_header));
  f.write(reinterpret_cast<const char *>(data), sizeof(fftw_complex) * m_no_of_pts);
}
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Save(std::vector<std::string> filenames, bool rescale) {
  if (rescale)
    for (int i = 0; i < no_wf; i++) {
      const double fak = sqrt(m_params->Get_VConstant("N", i));
      for (int l = 0; l < m_no_of_pts; l++) {
        m_Psi[i][l][0] *= fak;
        m_Psi[i][l][1] *= fak;
      }
    }
  for (int i = 0; i < no_wf; i++) Save(m_Psi[i], filenames[i]);
}
template <class T, int dim, int no_wf>
void CSOB_Base<T, dim, no_wf>::Save_Zero() {
  std::memset(m_Psi_sob[0], 0, sizeof(fftw_complex) * m_no_of_pts);
  Save(m_Psi_sob[0], "zero.bin");
}

template <class T, int dim, int no_wf>
ofstream &operator<<(ofstream &stream, CSOB_Base<T, dim, no_wf> &obj) {
  obj.Dump_2(stream);
  return stream;
}

#endif
