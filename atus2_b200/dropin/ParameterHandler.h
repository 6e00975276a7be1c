// ParameterHandler.h (drop-in) -- the XML program description of ATUS-2
// (source/libs/lib_myutils/ParameterHandler.h:17-103) for programs built
// against libatus_gpu.so: the same keys, defaults, sequence attributes and
// accessors, read by the engine's own XML reader (host/params.h).  Missing
// keys throw std::string as the reference's accessors do.
#ifndef ATUS_DROPIN_PARAMETERHANDLER_H
#define ATUS_DROPIN_PARAMETERHANDLER_H

#include <map>
#include <string>
#include <vector>

#include "../host/params.h"
#include "muParser.h"
#include "my_structs.h"

using atus::freq;
using atus::none;
using atus::each;
using atus::last;
using atus::packed;
typedef atus::sequence_item sequence_item;

struct analyze_item {
  std::string name;
  bool content;
  bool separate;
};

class ParameterHandler : public atus::ParameterHandler {
 public:
  explicit ParameterHandler(const std::string &filename) : atus::ParameterHandler(filename) {}

  std::string Get_simulation(const std::string &k) const { return atus::ParameterHandler::Get_simulation(k); }
  // muParser set-up of the programs: the CONSTANTS section plus Heaviside,
  // rect and sign (ParameterHandler.cpp:298-312)
  void Setup_muParser(mu::Parser &p) const {
    p.ClearConst();
    for (auto &c : constants()) p.DefineConst(c.first, c.second);
    p.DefineFun("Heaviside", atus::atus_heaviside, false);
    p.DefineFun("rect", atus::atus_rect, false);
    p.DefineFun("sign", atus::atus_sign, false);
  }
  // momentum states of component `comp` as "kx,ky,kz;..." (not read by the
  // programs this engine runs; kept for the interface)
  bool Get_MomentumStates(std::vector<double> &, const int) { return false; }

  std::vector<analyze_item> m_analyze;
  std::vector<zernike_polynomial> m_zernike;
};

#endif
