// bragg_ds -- Bragg beam splitter for two species of two internal states each
// (ATUS-2's bragg_ds, source/interferometry/src/bragg_ds.cpp) on the GPU engine.
//
//   bragg_ds run.xml
//
// Sequences: bragg_ad (one 2x2 Bragg exponential per species, each with its
// own laser and pulse window, on the GPU), freeprop (two-species IF potential
// step, on the GPU), freeprop_lin (kinetic steps only), set_momentum.  Rabi
// sums of species 1 in the bins {0, +-2 laser_k}, of species 2 in {0, +-2
// laser_k_2}, along x.
#include <omp.h>

#include "../solver.h"

using namespace atus;

template <int dim>
class Bragg_ds : public CRT_Base_IF_2<dim, 4> {
 public:
  explicit Bragg_ds(ParameterHandler *p) : CRT_Base_IF_2<dim, 4>(p) {
    this->m_gpu_steps["bragg_ad"] = ATUS_STEP_BRAGG_DS_AD;
    CPoint<dim> p1{}, p2{}, p3{};  // bragg_ds.cpp:73-90
    p2[0] = 2 * this->laser_k[0];
    p3[0] = -2 * this->laser_k[0];
    this->m_rabi_momentum_list.push_back(p1);
    this->m_rabi_momentum_list.push_back(p2);
    this->m_rabi_momentum_list.push_back(p3);
    p2[0] = 2 * this->laser_k2[0];
    p3[0] = -2 * this->laser_k2[0];
    this->m_rabi_momentum_list2.push_back(p1);
    this->m_rabi_momentum_list2.push_back(p2);
    this->m_rabi_momentum_list2.push_back(p3);
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
      Bragg_ds<1> s(&params);
      s.run_sequence();
    } else if (dim == 2) {
      Bragg_ds<2> s(&params);
      s.run_sequence();
    } else if (dim == 3) {
      Bragg_ds<3> s(&params);
      s.run_sequence();
    }
  } catch (std::string &str) {
    std::cout << str << std::endl;
  } catch (std::exception &e) {
    std::cout << e.what() << std::endl;
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
