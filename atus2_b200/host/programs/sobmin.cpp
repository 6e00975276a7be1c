// sobmin -- ground state by Sobolev-gradient descent (ATUS-2's sobmin,
// source/SOLVER/src/sob_solver.cpp) on the GPU engine.
//
//   sobmin run.xml        (ATUS_SOB_QUIET=1 silences the per-iteration lines)
//
// Grid from ALGORITHM, GUESS_<dim>D and POTENTIAL_<dim>D, Alpha_1, GS_1, N,
// epsilon and stepsize from the XML; writes FILENAME rescaled by sqrt(N) and
// zero.bin as the reference does.
#include <omp.h>

#include "../solver.h"

using namespace atus;

template <int dim>
class CSOB_Min : public CSOB_Base<dim, 1> {
 public:
  explicit CSOB_Min(ParameterHandler *p) : CSOB_Base<dim, 1>(p) {
    fill(this->m_params->Get_simulation("GUESS_" + std::to_string(dim) + "D"), true);
    fill(this->m_params->Get_simulation("POTENTIAL_" + std::to_string(dim) + "D"), false);
  }

 private:
  // Setup_Guess / Setup_Potential (sob_solver.cpp:63-150)
  void fill(const std::string &expr, bool guess) {
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
        if (guess) {
          this->m_Psi[0][2 * l] = e.Eval();
          this->m_Psi[0][2 * l + 1] = 0;
        } else {
          this->m_Potential[0][l] = e.Eval();
        }
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
    std::vector<std::string> filenames{params.Get_simulation("FILENAME")};
    if (dim == 1) {
      CSOB_Min<1> s(&params);
      s.run();
      s.Save(filenames, true);
      s.Save_Zero();
    } else if (dim == 2) {
      CSOB_Min<2> s(&params);
      s.run();
      s.Save(filenames, true);
      s.Save_Zero();
    } else if (dim == 3) {
      CSOB_Min<3> s(&params);
      s.run();
      s.Save(filenames, true);
      s.Save_Zero();
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
