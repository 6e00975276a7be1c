// bragg -- two-state Bragg beam splitter (ATUS-2's bragg,
// source/interferometry/src/bragg.cpp) on the GPU engine.
//
//   bragg run.xml
//
// Sequences: bragg_ad (analytic 2x2 exponential, on the GPU), freeprop (IF
// potential step, on the GPU), set_momentum, set_mirror (reads a mirror .bin),
// bragg_simple (the reference's constant-coupling step, on the host copy).
#include <omp.h>

#include <cstring>

#include "../solver.h"

using namespace atus;

template <int dim>
class Bragg_single : public CRT_Base_IF<dim, 2> {
 public:
  explicit Bragg_single(ParameterHandler *p) : CRT_Base_IF<dim, 2>(p) {
    this->m_gpu_steps["bragg_ad"] = ATUS_STEP_BRAGG_AD;
    this->m_map_stepfcts["bragg_simple"] = &Do_Bragg_simple_Wrapper;
    // Rabi momentum bins {0, +2 laser_k, -2 laser_k} along x (bragg.cpp:85-93)
    CPoint<dim> p1{}, p2{}, p3{};
    p2[0] = 2 * this->laser_k[0];
    p3[0] = -2 * this->laser_k[0];
    this->m_rabi_momentum_list.push_back(p1);
    this->m_rabi_momentum_list.push_back(p2);
    this->m_rabi_momentum_list.push_back(p3);
    m_no_of_Mirror_pts = (int)(this->Get_dimY() * this->Get_dimZ());
    m_Mirror.assign(m_no_of_Mirror_pts, 0.0);
  }

 protected:
  bool check_consistency(const generic_header &head) {
    if (dim == 2) return head.nDimX == this->Get_dimY();
    if (dim == 3) return head.nDimX == this->Get_dimY() && head.nDimY == this->Get_dimZ();
    return false;
  }
  bool run_custom_sequence(const sequence_item &item) override {
    if (item.name == "set_mirror") {
      generic_header h{};
      std::ifstream f(item.content, std::ifstream::binary);
      f.read((char *)&h, sizeof(generic_header));
      if (check_consistency(h)) {
        f.seekg(sizeof(generic_header), std::ifstream::beg);
        f.read((char *)m_Mirror.data(), sizeof(double) * m_no_of_Mirror_pts);
      } else {
        std::cout << "Change number of points for mirror." << std::endl;
        exit(EXIT_FAILURE);
      }
      return true;
    }
    return false;
  }

  static void Do_Bragg_simple_Wrapper(void *ptr, sequence_item &) { static_cast<Bragg_single *>(ptr)->Do_Bragg_simple(); }

  // Constant-coupling two-level step (bragg.cpp:306-371), on the host copy.
  void Do_Bragg_simple() {
    const double dt = this->Get_dt();
    fftw_complex *P1 = reinterpret_cast<fftw_complex *>(this->m_fields[0].data());
    fftw_complex *P2 = reinterpret_cast<fftw_complex *>(this->m_fields[1].data());
    const double Omega = -this->Amp[0] * this->Amp[0] / (4 * this->DeltaL[1]);
    const double om0 = std::cos(2 * Omega * dt), om1 = std::sin(2 * Omega * dt);
    const double ph0 = 1.0, ph1 = 0.0;  // phase1 = 0
    const double O11[2] = {0.5 * (1 + om0), 0.5 * om1};
    const double O22[2] = {O11[0], O11[1]};
    const double O12[2] = {0.5 * (ph0 * om0 - ph0 - ph1 * om1), 0.5 * (ph0 * om1 + ph1 * om0 - ph1)};
    const double O21[2] = {0.5 * (ph0 * om0 - ph0 + ph1 * om1), 0.5 * (ph0 * om1 - ph1 * om0 + ph1)};
    for (int64_t l = 0; l < this->m_grid.npts; l++) {
      const double g0 = P1[l][0], g1 = P1[l][1], m0 = P2[l][0], m1 = P2[l][1];
      P1[l][0] = (O11[0] * g0 - O11[1] * g1) + (O12[0] * m0 - O12[1] * m1);
      P1[l][1] = (O11[0] * g1 + O11[1] * g0) + (O12[0] * m1 + O12[1] * m0);
      P2[l][0] = (O21[0] * g0 - O21[1] * g1) + (O22[0] * m0 - O22[1] * m1);
      P2[l][1] = (O21[0] * g1 + O21[1] * g0) + (O22[0] * m1 + O22[1] * m0);
    }
  }

  std::vector<double> m_Mirror;
  int m_no_of_Mirror_pts = 0;
};

int main(int argc, char *argv[]) {
  if (argc != 2) {
    printf("No parameter xml file specified.\n");
    return EXIT_FAILURE;
  }
  try {
    ParameterHandler params(argv[1]);
    const int dim = std::stoi(params.Get_simulation("DIM"));
    int threads = 4;
    if (const char *env = getenv("MY_NO_OF_THREADS")) threads = atoi(env);
    omp_set_num_threads(threads);
    if (dim == 1) {
      Bragg_single<1> s(&params);
      s.run_sequence();
    } else if (dim == 2) {
      Bragg_single<2> s(&params);
      s.run_sequence();
    } else if (dim == 3) {
      Bragg_single<3> s(&params);
      s.run_sequence();
    } else {
      std::cout << "You have found a new dimension!" << std::endl;
    }
  } catch (std::string &str) {
    std::cout << str << std::endl;
    return EXIT_FAILURE;
  } catch (std::exception &e) {
    std::cout << e.what() << std::endl;
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
