// gen_psi_0 -- writes the initial wave function of an XML program
// (ATUS-2's gen_psi_0, source/utils/src/gen_psi_0.cpp): GUESS_<dim>D on the
// grid of the ALGORITHM section, x_i = (i - N/2) dx, normalised to the
// constant N, saved as FILENAME.  Host only.
#include <omp.h>

#include "../solver.h"

using namespace atus;

template <int dim>
static void generate(ParameterHandler &ph) {
  Grid<dim> g;
  generic_header &h = g.h;
  h = generic_header{};
  h.nDims = dim;
  h.nself = sizeof(generic_header);
  h.bAtom = 1;
  h.bComplex = 1;
  h.nDatatyp = 16;
  h.xMax = ph.Get_xMax();
  h.xMin = ph.Get_xMin();
  h.yMax = ph.Get_yMax();
  h.yMin = ph.Get_yMin();
  h.zMax = ph.Get_zMax();
  h.zMin = ph.Get_zMin();
  h.dt = 0.001;
  h.nDimX = ph.Get_NX();
  h.nDimY = dim >= 2 ? ph.Get_NY() : 1;
  h.nDimZ = dim >= 3 ? ph.Get_NZ() : 1;
  h.dx = std::fabs(h.xMax - h.xMin) / double(h.nDimX);
  h.dkx = 2 * M_PI / std::fabs(h.xMax - h.xMin);
  if (dim >= 2) {
    h.dy = std::fabs(h.yMax - h.yMin) / double(h.nDimY);
    h.dky = 2 * M_PI / std::fabs(h.yMax - h.yMin);
  }
  if (dim >= 3) {
    h.dz = std::fabs(h.zMax - h.zMin) / double(h.nDimZ);
    h.dkz = 2 * M_PI / std::fabs(h.zMax - h.zMin);
  }
  g.setup();
  const std::string filename = ph.Get_simulation("FILENAME");
  const std::string guess = ph.Get_simulation("GUESS_" + std::to_string(dim) + "D");
  const double n_particles = ph.Get_Constant("N");
  std::vector<double> psi(2 * g.npts, 0.0);
  double N = 0;
  #pragma omp parallel
  {
    CPoint<dim> x{};
    Expr e;
    ph.Setup_Parser(e);
    e.SetExpr(guess);
    const char *names[3] = {"x", "y", "z"};
    for (int a = 0; a < dim; a++) e.DefineVar(names[a], &x[a]);
    #pragma omp for reduction(+ : N)
    for (int64_t l = 0; l < g.npts; l++) {
      x = g.Get_x(l);
      psi[2 * l] = e.Eval();
      N += psi[2 * l] * psi[2 * l];
    }
  }
  N *= g.ar;
  if (N > 0.0) {
    const double f = std::sqrt(n_particles / N);
    for (int64_t l = 0; l < g.npts; l++) psi[2 * l] *= f;
  }
  std::ofstream ofs(filename, std::ofstream::binary);
  ofs.write((const char *)&h, sizeof(generic_header));
  ofs.write((const char *)psi.data(), 16 * g.npts);
}

int main(int argc, char *argv[]) {
  if (argc != 2) {
    printf("No xml file specified.\n");
    return EXIT_FAILURE;
  }
  try {
    ParameterHandler params(argv[1]);
    const int dim = std::stoi(params.Get_simulation("DIM"));
    std::cout << "DIM = " << dim << std::endl;
    if (dim == 1) generate<1>(params);
    if (dim == 2) generate<2>(params);
    if (dim == 3) generate<3>(params);
  } catch (std::string &str) {
    std::cout << str << std::endl;
    return EXIT_FAILURE;
  } catch (std::exception &e) {
    std::cout << e.what() << std::endl;
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
