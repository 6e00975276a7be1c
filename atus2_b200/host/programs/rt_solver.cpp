// rt_solver -- real-time propagation of one component (ATUS-2's rt_solver,
// source/SOLVER/src/rt_solver.cpp) on the GPU engine.
//
//   rt_solver run.xml
//
// Reads FILENAME (.bin), POTENTIAL_<dim>D, Alpha_1, GS_1 and the SEQUENCE
// exactly as the reference program does and writes the same files and
// console lines; the propagation runs through libatus_gpu.so.
#include <omp.h>

#include "../solver.h"

using namespace atus;

template <int dim>
class CRT_Propagation : public CRT_Base<dim, 1> {
 public:
  explicit CRT_Propagation(ParameterHandler *p) : CRT_Base<dim, 1>(p) {
    this->Init_Potential();
    Setup_Potential();
  }

 protected:
  bool run_custom_sequence(const sequence_item &) override { return false; }

  // V on the grid from POTENTIAL_<dim>D (rt_solver.cpp:73-131).
  void Setup_Potential() {
    const std::string expr = this->m_params->Get_simulation("POTENTIAL_" + std::to_string(dim) + "D");
    const int64_t n = this->m_grid.npts;
    #pragma omp parallel
    {
      CPoint<dim> x{};
      Expr e;
      this->m_params->Setup_Parser(e);
      e.SetExpr(expr);
      const char *names[3] = {"x", "y", "z"};
      for (int a = 0; a < dim; a++) e.DefineVar(names[a], &x[a]);
      #pragma omp for
      for (int64_t l = 0; l < n; l++) {
        x = this->m_grid.Get_x(l);
        this->m_Potential[0][l] = e.Eval();
      }
    }
    this->m_pot_dirty = true;
    if (dim == 2) {
      std::ofstream outf("potential.txt");
      for (int i = 0; i < this->Get_dimX(); i++) {
        const double x = double(i - this->m_grid.shift[0]) * this->m_grid.h.dx;
        for (int j = 0; j < this->Get_dimY(); j++) {
          const double y = double(j - this->m_grid.shift[1]) * this->m_grid.h.dy;
          outf << x << "\t" << y << "\t" << this->m_Potential[0][j + this->Get_dimY() * i] << "\n";
        }
        outf << "\n";
      }
    }
  }
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
      CRT_Propagation<1> s(&params);
      s.run_sequence();
    } else if (dim == 2) {
      CRT_Propagation<2> s(&params);
      s.run_sequence();
    } else if (dim == 3) {
      CRT_Propagation<3> s(&params);
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
