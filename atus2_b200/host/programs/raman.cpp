// raman -- three-state Raman beam splitter (ATUS-2's raman,
// source/interferometry/src/raman.cpp) on the GPU engine.
//
//   raman run.xml
//
// Sequences: raman (three-state Raman exponential of Numerical_Raman, on the
// GPU), bragg (n-state exponential of Numerical_Bragg, on the GPU), freeprop
// (IF potential step, on the GPU), set_momentum.  Rabi sums in the momentum
// bins {0, +2 laser_k, -2 laser_k} along x.
#include <omp.h>

#include "../solver.h"

using namespace atus;

template <int dim>
class Raman_single : public CRT_Base_IF<dim, 3> {
 public:
  explicit Raman_single(ParameterHandler *p) : CRT_Base_IF<dim, 3>(p) {
    CPoint<dim> p1{}, p2{}, p3{};  // raman.cpp:56-67
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
      Raman_single<1> s(&params);
      s.run_sequence();
    } else if (dim == 2) {
      Raman_single<2> s(&params);
      s.run_sequence();
    } else if (dim == 3) {
      Raman_single<3> s(&params);
      s.run_sequence();
    } else {
      std::cout << "You have found a new dimension!" << std::endl;
    }
  } catch (std::string &str) {
    std::cout << str << std::endl;
  } catch (std::exception &e) {
    std::cout << e.what() << std::endl;
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
