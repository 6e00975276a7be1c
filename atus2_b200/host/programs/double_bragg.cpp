// double_bragg -- three-state (double) Bragg beam splitter (ATUS-2's
// double_bragg, source/interferometry/src/double_bragg.cpp) on the GPU engine.
//
//   double_bragg run.xml
//
// Sequences: bragg_ad (the three-level exponential of Do_Double_Bragg_ad, on
// the GPU) and freeprop (IF potential step, on the GPU); Rabi sums in the
// momentum bins {0, +2 laser_k, -2 laser_k} along x.
#include <omp.h>

#include "../solver.h"

using namespace atus;

template <int dim>
class Bragg_double : public CRT_Base_IF<dim, 3> {
 public:
  explicit Bragg_double(ParameterHandler *p) : CRT_Base_IF<dim, 3>(p) {
    this->m_gpu_steps["bragg_ad"] = ATUS_STEP_DOUBLE_BRAGG_AD;
    CPoint<dim> p1{}, p2{}, p3{};  // double_bragg.cpp:76-84
    p2[0] = 2 * this->laser_k[0];
    p3[0] = -2 * this->laser_k[0];
    this->m_rabi_momentum_list.push_back(p1);
    this->m_rabi_momentum_list.push_back(p2);
    this->m_rabi_momentum_list.push_back(p3);
  }

 protected:
  bool run_custom_sequence(const sequence_item &) override { return false; }
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
      Bragg_double<1> s(&params);
      s.run_sequence();
    } else if (dim == 2) {
      Bragg_double<2> s(&params);
      s.run_sequence();
    } else if (dim == 3) {
      Bragg_double<3> s(&params);
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
