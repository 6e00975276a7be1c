// params.h -- the XML program description of ATUS-2 (SIMULATION files).
//
// ParameterHandler reads the same file layout, with the same keys, defaults
// and sequence attributes, as the reference's ParameterHandler
// (source/libs/lib_myutils/ParameterHandler.cpp:14-563):
//   <SIMULATION>  direct children with text    -> Get_simulation(key)
//   CONSTANTS//*  name -> double               -> Get_Constant
//   VCONSTANTS//* name -> comma-separated list -> Get_VConstant(key[, i])
//   ALGORITHM//*  NX.. XMIN.. DT, EPSILON ...  -> Get_NX(), Get_dt(), ...
//   SEQUENCE//*   one sequence_item per element (dt, Nk, *_freq, chirps)
// The XML reader is a small recursive-descent parser for this subset
// (elements, attributes, text, comments, declarations).
#pragma once

#include <cmath>
#include <cstdint>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "expr.h"
#include "my_structs.h"

namespace atus {

struct XmlNode {
  std::string name, text;
  std::map<std::string, std::string> attr;
  std::vector<std::unique_ptr<XmlNode>> kids;
};

class XmlReader {
 public:
  static std::unique_ptr<XmlNode> parse_file(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("Critical error occured during loading of file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    XmlReader r(ss.str());
    return r.document();
  }

 private:
  explicit XmlReader(std::string s) : s_(std::move(s)) {}
  std::unique_ptr<XmlNode> document() {
    skip_misc();
    if (i_ >= s_.size() || s_[i_] != '<') throw std::runtime_error("xml: no root element");
    auto root = element();
    return root;
  }
  void skip_ws() {
    while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) i_++;
  }
  bool starts(const char *p) const { return s_.compare(i_, std::char_traits<char>::length(p), p) == 0; }
  void skip_until(const char *end) {
    size_t j = s_.find(end, i_);
    if (j == std::string::npos) throw std::runtime_error(std::string("xml: unterminated, expected ") + end);
    i_ = j + std::char_traits<char>::length(end);
  }
  void skip_misc() {
    for (;;) {
      skip_ws();
      if (starts("<?")) skip_until("?>");
      else if (starts("<!--")) skip_until("-->");
      else if (starts("<!")) skip_until(">");
      else return;
    }
  }
  std::string name() {
    size_t j = i_;
    while (j < s_.size() && (std::isalnum((unsigned char)s_[j]) || s_[j] == '_' || s_[j] == '-' || s_[j] == '.' || s_[j] == ':')) j++;
    if (j == i_) throw std::runtime_error("xml: expected a name at offset " + std::to_string(i_));
    std::string n = s_.substr(i_, j - i_);
    i_ = j;
    return n;
  }
  static std::string unescape(const std::string &t) {
    std::string o;
    for (size_t k = 0; k < t.size(); k++) {
      if (t[k] == '&') {
        static const std::pair<const char *, char> ents[] = {{"&lt;", '<'}, {"&gt;", '>'}, {"&amp;", '&'}, {"&quot;", '"'}, {"&apos;", '\''}};
        bool done = false;
        for (auto &e : ents) {
          const size_t L = std::char_traits<char>::length(e.first);
          if (t.compare(k, L, e.first) == 0) { o += e.second; k += L - 1; done = true; break; }
        }
        if (!done) o += t[k];
      } else {
        o += t[k];
      }
    }
    return o;
  }
  std::unique_ptr<XmlNode> element() {
    i_++;  // '<'
    auto n = std::make_unique<XmlNode>();
    n->name = name();
    for (;;) {
      skip_ws();
      if (starts("/>")) { i_ += 2; return n; }
      if (starts(">")) { i_++; break; }
      std::string an = name();
      skip_ws();
      if (i_ >= s_.size() || s_[i_] != '=') throw std::runtime_error("xml: expected '=' after attribute " + an);
      i_++;
      skip_ws();
      const char q = s_[i_];
      if (q != '"' && q != '\'') throw std::runtime_error("xml: unquoted attribute " + an);
      size_t j = s_.find(q, i_ + 1);
      if (j == std::string::npos) throw std::runtime_error("xml: unterminated attribute " + an);
      n->attr[an] = unescape(s_.substr(i_ + 1, j - i_ - 1));
      i_ = j + 1;
    }
    for (;;) {
      if (i_ >= s_.size()) throw std::runtime_error("xml: unterminated element " + n->name);
      if (starts("<!--")) { skip_until("-->"); continue; }
      if (starts("</")) {
        i_ += 2;
        std::string en = name();
        if (en != n->name) throw std::runtime_error("xml: </" + en + "> closes <" + n->name + ">");
        skip_ws();
        if (s_[i_] != '>') throw std::runtime_error("xml: bad closing tag " + en);
        i_++;
        return n;
      }
      if (s_[i_] == '<') { n->kids.push_back(element()); continue; }
      size_t j = s_.find('<', i_);
      if (j == std::string::npos) j = s_.size();
      n->text += unescape(s_.substr(i_, j - i_));
      i_ = j;
    }
  }
  std::string s_;
  size_t i_ = 0;
};

enum freq { none = 0, each = 1, last = 2, packed = 3 };

// One element of <SEQUENCE> (ParameterHandler.h:17-35, defaults of
// ParameterHandler.cpp:63-86).
struct sequence_item {
  std::string name, content;
  std::vector<double> duration;
  double dt = 0.001;
  double chirp_min = 0, chirp_max = 0;
  int no_of_chirps = 1, chirp_mode = 0;
  int rabi_output_freq = none, output_freq = none, custom_freq = none;
  int comp = 0, compute_pn_freq = last, analyze = none, Nk = 100;
  double time = 0;
};

class ParameterHandler {
 public:
  explicit ParameterHandler(const std::string &filename) {
    root_ = XmlReader::parse_file(filename);
    if (root_->name != "SIMULATION") throw std::runtime_error("root element must be <SIMULATION> in " + filename);
    for (auto &k : root_->kids)
      if (k->kids.empty()) m_simulation[k->name] = trim_keep(k->text);
    for (const XmlNode *sec : sections("CONSTANTS"))
      for (const XmlNode *e : descendants(sec)) {
        try {
          m_constants[e->name] = std::stod(e->text);
        } catch (const std::exception &) {
          throw std::runtime_error("Error Parsing xml file: Unable to convert " + e->text + " to double for element <" +
                                   e->name + "> in section CONSTANTS");
        }
      }
    for (const XmlNode *sec : sections("VCONSTANTS"))
      for (const XmlNode *e : descendants(sec)) {
        std::vector<double> v;
        for (const std::string &p : split(e->text)) {
          try {
            v.push_back(std::stod(p));
          } catch (const std::exception &) {
            throw std::runtime_error("Error Parsing xml file: Unable to convert " + e->text + " to double for element <" +
                                     e->name + "> in section VCONSTANTS");
          }
        }
        m_vconstants[e->name] = v;
      }
    for (const XmlNode *sec : sections("ALGORITHM"))
      for (const XmlNode *e : descendants(sec)) m_algorithm[e->name] = e->text;
    for (const XmlNode *sec : sections("SEQUENCE"))
      for (const XmlNode *e : descendants(sec)) m_sequence.push_back(item(*e));
  }

  std::string Get_simulation(const std::string &k) const {
    auto it = m_simulation.find(k);
    if (it == m_simulation.end()) throw std::string("Error: Could not find the key: " + k + " in section SIMULATION.");
    return it->second;
  }
  bool Has_simulation(const std::string &k) const { return m_simulation.count(k) != 0; }
  const std::map<std::string, double> &constants() const { return m_constants; }
  double Get_Constant(const std::string &k) const {
    auto it = m_constants.find(k);
    if (it == m_constants.end()) throw std::string("Error: Could not find the key: " + k + " in section CONSTANT.");
    return it->second;
  }
  double Get_VConstant(const std::string &k, int p) const {
    auto it = m_vconstants.find(k);
    if (it == m_vconstants.end()) throw std::string("Error: Could not find the key " + k + " in section VCONSTANTS.");
    if (p < 0 || p >= (int)it->second.size())
      throw std::string("Error: element " + std::to_string(p) + " of " + k + " is missing in section VCONSTANTS.");
    return it->second[p];
  }
  std::vector<double> Get_VConstant(const std::string &k) const {
    auto it = m_vconstants.find(k);
    if (it == m_vconstants.end()) throw std::string("Error: Could not find the key " + k + " in section VCONSTANTS.");
    return it->second;
  }

  double Get_dt() const { return algo_d("DT", 0.001); }
  double Get_t() const { return algo_d("T", 0); }
  double Get_epsilon() const { return algo_d("EPSILON", 1e-5); }
  double Get_stepsize() const { return algo_d("STEPSIZE", 0.001); }
  double Get_xMax() const { return algo_d("XMAX", 10.0); }
  double Get_xMin() const { return algo_d("XMIN", -10.0); }
  double Get_yMax() const { return algo_d("YMAX", 10.0); }
  double Get_yMin() const { return algo_d("YMIN", -10.0); }
  double Get_zMax() const { return algo_d("ZMAX", 10.0); }
  double Get_zMin() const { return algo_d("ZMIN", -10.0); }
  int Get_NX() const { return algo_i("NX", 256); }
  int Get_NY() const { return algo_i("NY", 256); }
  int Get_NZ() const { return algo_i("NZ", 256); }
  int Get_NA() const { return algo_i("NA", 10); }
  int Get_NK() const { return algo_i("NK", 10); }
  int Get_MaxIter() const { return algo_i("MAXITER", 10); }

  // Header of the grid the ALGORITHM section describes
  // (ParameterHandler::Get_Header, ParameterHandler.cpp:488-563).
  void Get_Header(generic_header &h, bool bcomplex = true) const {
    h = generic_header{};
    const long long nDims = (long long)std::stod(Get_simulation("DIM"));
    h.nself = sizeof(generic_header);
    h.nDatatyp = bcomplex ? 16 : 8;
    h.bComplex = bcomplex ? 1 : 0;
    h.bAtom = 1;
    h.nDims = nDims;
    h.nDimX = Get_NX();
    h.nDimY = nDims >= 2 ? Get_NY() : 1;
    h.nDimZ = nDims >= 3 ? Get_NZ() : 1;
    h.xMax = Get_xMax();
    h.xMin = Get_xMin();
    h.dx = std::fabs(h.xMax - h.xMin) / double(h.nDimX);
    h.dkx = 2 * M_PI / std::fabs(h.xMax - h.xMin);
    if (nDims >= 2) {
      h.yMax = Get_yMax();
      h.yMin = Get_yMin();
      h.dy = std::fabs(h.yMax - h.yMin) / double(h.nDimY);
      h.dky = 2 * M_PI / std::fabs(h.yMax - h.yMin);
    }
    if (nDims >= 3) {
      h.zMax = Get_zMax();
      h.zMin = Get_zMin();
      h.dz = std::fabs(h.zMax - h.zMin) / double(h.nDimZ);
      h.dkz = 2 * M_PI / std::fabs(h.zMax - h.zMin);
    }
    h.dt = 0.001;
    h.nself_and_data = h.nself + (h.nDimX + h.nDimY) * h.nDatatyp;
  }

  // Constants plus Heaviside, rect and sign, as Setup_muParser provides them.
  void Setup_Parser(Expr &e) const {
    e.ClearConst();
    for (auto &c : m_constants) e.DefineConst(c.first, c.second);
    e.DefineFun("Heaviside", atus_heaviside);
    e.DefineFun("rect", atus_rect);
    e.DefineFun("sign", atus_sign);
  }

  std::vector<sequence_item> m_sequence;

 private:
  static std::string trim_keep(const std::string &t) { return t; }
  static std::vector<std::string> split(const std::string &t) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : t) {
      if (ch == ',') { out.push_back(cur); cur.clear(); }
      else cur += ch;
    }
    out.push_back(cur);
    // drop surrounding blanks of every part
    for (auto &p : out) {
      size_t a = p.find_first_not_of(" \t\r\n"), b = p.find_last_not_of(" \t\r\n");
      p = (a == std::string::npos) ? std::string() : p.substr(a, b - a + 1);
    }
    return out;
  }
  static void collect(const XmlNode *n, std::vector<const XmlNode *> &out) {
    for (auto &k : n->kids) {
      out.push_back(k.get());
      collect(k.get(), out);
    }
  }
  static std::vector<const XmlNode *> descendants(const XmlNode *n) {
    std::vector<const XmlNode *> v;
    collect(n, v);
    return v;
  }
  std::vector<const XmlNode *> sections(const std::string &name) const {
    std::vector<const XmlNode *> all, out;
    collect(root_.get(), all);
    for (auto *n : all)
      if (n->name == name) out.push_back(n);
    return out;
  }
  static int freq_of(const XmlNode &e, const char *a, const char *def) {
    auto it = e.attr.find(a);
    const std::string v = it == e.attr.end() ? def : it->second;
    if (v == "each") return each;
    if (v == "last") return last;
    if (v == "packed") return packed;
    return none;
  }
  static double attr_d(const XmlNode &e, const char *a, double def) {
    auto it = e.attr.find(a);
    if (it == e.attr.end()) return def;
    try { return std::stod(it->second); } catch (const std::exception &) { return def; }
  }
  static int attr_i(const XmlNode &e, const char *a, int def) {
    auto it = e.attr.find(a);
    if (it == e.attr.end()) return def;
    try { return std::stoi(it->second); } catch (const std::exception &) { return def; }
  }
  static sequence_item item(const XmlNode &e) {
    sequence_item s;
    s.name = e.name;
    s.content = e.text;
    s.dt = attr_d(e, "dt", 0.001);
    s.Nk = attr_i(e, "Nk", 100);
    s.comp = attr_i(e, "comp", 0);
    s.output_freq = freq_of(e, "output_freq", "none");
    s.rabi_output_freq = freq_of(e, "rabi_output_freq", "none");
    s.compute_pn_freq = freq_of(e, "pn_freq", "last");
    s.custom_freq = freq_of(e, "custom_freq", "none");
    s.analyze = freq_of(e, "analyze", "none");
    s.chirp_mode = attr_i(e, "chirp_mode", 0);
    s.no_of_chirps = attr_i(e, "no_of_chirps", 1);
    s.chirp_min = attr_d(e, "chirp_min", 0);
    s.chirp_max = attr_d(e, "chirp_max", 0);
    for (const std::string &p : split(e.text)) {
      double v = 0.0;
      try { v = std::stod(p); } catch (const std::exception &) { v = 0.0; }
      s.duration.push_back(v);
    }
    return s;
  }
  double algo_d(const char *k, double def) const {
    auto it = m_algorithm.find(k);
    return it == m_algorithm.end() ? def : std::stod(it->second);
  }
  int algo_i(const char *k, int def) const {
    auto it = m_algorithm.find(k);
    return it == m_algorithm.end() ? def : std::stoi(it->second);
  }

  std::unique_ptr<XmlNode> root_;
  std::map<std::string, std::string> m_simulation, m_algorithm;
  std::map<std::string, double> m_constants;
  std::map<std::string, std::vector<double>> m_vconstants;
};

}  // namespace atus
