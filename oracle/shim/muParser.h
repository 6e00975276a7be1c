/*
 * muParser.h -- the subset of the muParser 2.2.6 API the reference programs use,
 * for building them in the oracle (test infrastructure only; muParser itself is
 * not installed here).
 *
 * Used by ParameterHandler::Setup_muParser (ParameterHandler.cpp:298-312),
 * rt_solver.cpp:79-113, sob_solver.cpp:73-137, CRT_Base_IF.h:178-184 and
 * gen_psi_0.cpp:125-154: SetExpr, DefineVar, DefineConst, DefineFun (1- and
 * 3-argument), ClearConst, Eval and mu::Parser::exception_type with
 * GetMsg/GetExpr/GetToken/GetPos/GetCode.
 *
 * Grammar and precedence follow muParser's documented rules: ?: < || < && <
 * comparisons < + - < * / < unary sign < ^ (right associative), so -x^2 is
 * -(x^2).  Built-ins: sin cos tan asin acos atan sinh cosh tanh asinh acosh
 * atanh exp log ln log2 log10 sqrt abs sign rint min max, constants _pi _e.
 * The expression is compiled to a postfix program once and evaluated with a
 * small value stack; ^ is evaluated with pow().
 */
#ifndef ORACLE_SHIM_MUPARSER_H
#define ORACLE_SHIM_MUPARSER_H

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

namespace mu {

typedef double value_type;
typedef std::string string_type;

class ParserError {
 public:
  ParserError(const std::string &msg, const std::string &expr, const std::string &tok, int pos, int code)
      : m_msg(msg), m_expr(expr), m_tok(tok), m_pos(pos), m_code(code) {}
  const std::string &GetMsg() const { return m_msg; }
  const std::string &GetExpr() const { return m_expr; }
  const std::string &GetToken() const { return m_tok; }
  int GetPos() const { return m_pos; }
  int GetCode() const { return m_code; }

 private:
  std::string m_msg, m_expr, m_tok;
  int m_pos, m_code;
};

class Parser {
 public:
  typedef ParserError exception_type;
  typedef double (*fun1_t)(double);
  typedef double (*fun2_t)(double, double);
  typedef double (*fun3_t)(double, double, double);

  Parser() : m_dirty(true) {}

  void SetExpr(const std::string &e) { m_expr = e; m_dirty = true; }
  void DefineVar(const std::string &n, double *p) { m_vars[n] = p; m_dirty = true; }
  void DefineConst(const std::string &n, double v) { m_consts[n] = v; m_dirty = true; }
  void ClearConst() { m_consts.clear(); m_dirty = true; }
  void ClearVar() { m_vars.clear(); m_dirty = true; }
  void DefineFun(const std::string &n, fun1_t f, bool = true) { m_f1[n] = f; m_dirty = true; }
  void DefineFun(const std::string &n, fun2_t f, bool = true) { m_f2[n] = f; m_dirty = true; }
  void DefineFun(const std::string &n, fun3_t f, bool = true) { m_f3[n] = f; m_dirty = true; }
  const std::string &GetExpr() const { return m_expr; }

  double Eval() const {
    if (m_dirty) compile();
    double st[64];
    int sp = 0;
    for (const Ins &in : m_prog) {
      switch (in.op) {
        case PUSH: st[sp++] = in.v; break;
        case VAR: st[sp++] = *in.p; break;
        case NEG: st[sp - 1] = -st[sp - 1]; break;
        case ADD: sp--; st[sp - 1] = st[sp - 1] + st[sp]; break;
        case SUB: sp--; st[sp - 1] = st[sp - 1] - st[sp]; break;
        case MUL: sp--; st[sp - 1] = st[sp - 1] * st[sp]; break;
        case DIV: sp--; st[sp - 1] = st[sp - 1] / st[sp]; break;
        case POW: sp--; st[sp - 1] = std::pow(st[sp - 1], st[sp]); break;
        case LT: sp--; st[sp - 1] = st[sp - 1] < st[sp]; break;
        case GT: sp--; st[sp - 1] = st[sp - 1] > st[sp]; break;
        case LE: sp--; st[sp - 1] = st[sp - 1] <= st[sp]; break;
        case GE: sp--; st[sp - 1] = st[sp - 1] >= st[sp]; break;
        case EQ: sp--; st[sp - 1] = st[sp - 1] == st[sp]; break;
        case NE: sp--; st[sp - 1] = st[sp - 1] != st[sp]; break;
        case AND: sp--; st[sp - 1] = (st[sp - 1] != 0) && (st[sp] != 0); break;
        case OR: sp--; st[sp - 1] = (st[sp - 1] != 0) || (st[sp] != 0); break;
        case SEL: sp -= 2; st[sp - 1] = (st[sp - 1] != 0) ? st[sp] : st[sp + 1]; break;
        case F1: st[sp - 1] = in.f1(st[sp - 1]); break;
        case F2: sp--; st[sp - 1] = in.f2(st[sp - 1], st[sp]); break;
        case F3: sp -= 2; st[sp - 1] = in.f3(st[sp - 1], st[sp], st[sp + 1]); break;
      }
    }
    return st[0];
  }

 private:
  enum Op { PUSH, VAR, NEG, ADD, SUB, MUL, DIV, POW, LT, GT, LE, GE, EQ, NE, AND, OR, SEL, F1, F2, F3 };
  struct Ins {
    Op op;
    double v;
    const double *p;
    fun1_t f1;
    fun2_t f2;
    fun3_t f3;
  };

  static double b_sign(double x) { return (x > 0) ? 1.0 : ((x < 0) ? -1.0 : 0.0); }
  static double b_min(double a, double b) { return a < b ? a : b; }
  static double b_max(double a, double b) { return a > b ? a : b; }
  static double b_log(double x) { return std::log(x); }
  static double b_rint(double x) { return std::rint(x); }

  void fail(const std::string &msg, const std::string &tok) const {
    throw ParserError(msg, m_expr, tok, (int)m_pos, 1);
  }
  void emit(Op op) const { Ins i = {op, 0, nullptr, nullptr, nullptr, nullptr}; m_prog.push_back(i); }

  void skip() const {
    while (m_pos < m_expr.size() && std::isspace((unsigned char)m_expr[m_pos])) m_pos++;
  }
  bool accept(const char *s) const {
    skip();
    size_t n = std::char_traits<char>::length(s);
    if (m_expr.compare(m_pos, n, s) == 0) {
      m_pos += n;
      return true;
    }
    return false;
  }

  void compile() const {
    m_prog.clear();
    m_pos = 0;
    if (m_expr.find_first_not_of(" \t\r\n") == std::string::npos) fail("Unexpected end of expression", "");
    p_ternary();
    skip();
    if (m_pos != m_expr.size()) fail("Unexpected token", m_expr.substr(m_pos, 1));
    m_dirty = false;
  }

  void p_ternary() const {
    p_or();
    if (accept("?")) {
      p_ternary();
      if (!accept(":")) fail("Missing ':' in ternary", "");
      p_ternary();
      emit(SEL);
    }
  }
  void p_or() const {
    p_and();
    while (accept("||")) { p_and(); emit(OR); }
  }
  void p_and() const {
    p_cmp();
    while (accept("&&")) { p_cmp(); emit(AND); }
  }
  void p_cmp() const {
    p_add();
    for (;;) {
      if (accept("<=")) { p_add(); emit(LE); }
      else if (accept(">=")) { p_add(); emit(GE); }
      else if (accept("==")) { p_add(); emit(EQ); }
      else if (accept("!=")) { p_add(); emit(NE); }
      else if (accept("<")) { p_add(); emit(LT); }
      else if (accept(">")) { p_add(); emit(GT); }
      else break;
    }
  }
  void p_add() const {
    p_mul();
    for (;;) {
      if (accept("+")) { p_mul(); emit(ADD); }
      else if (accept("-")) { p_mul(); emit(SUB); }
      else break;
    }
  }
  void p_mul() const {
    p_unary();
    for (;;) {
      if (accept("*")) { p_unary(); emit(MUL); }
      else if (accept("/")) { p_unary(); emit(DIV); }
      else break;
    }
  }
  void p_unary() const {
    if (accept("-")) { p_unary(); emit(NEG); return; }
    if (accept("+")) { p_unary(); return; }
    p_pow();
  }
  void p_pow() const {
    p_primary();
    if (accept("^")) { p_unary(); emit(POW); }
  }
  void p_primary() const {
    skip();
    if (m_pos >= m_expr.size()) fail("Unexpected end of expression", "");
    const char ch = m_expr[m_pos];
    if (ch == '(') {
      m_pos++;
      p_ternary();
      if (!accept(")")) fail("Missing parenthesis", "");
      return;
    }
    if (std::isdigit((unsigned char)ch) || ch == '.') {
      const char *b = m_expr.c_str() + m_pos;
      char *e = nullptr;
      const double v = std::strtod(b, &e);
      if (e == b) fail("Invalid number", std::string(1, ch));
      m_pos += (size_t)(e - b);
      Ins i = {PUSH, v, nullptr, nullptr, nullptr, nullptr};
      m_prog.push_back(i);
      return;
    }
    if (std::isalpha((unsigned char)ch) || ch == '_') {
      size_t s = m_pos;
      while (m_pos < m_expr.size() && (std::isalnum((unsigned char)m_expr[m_pos]) || m_expr[m_pos] == '_')) m_pos++;
      const std::string name = m_expr.substr(s, m_pos - s);
      skip();
      if (m_pos < m_expr.size() && m_expr[m_pos] == '(') {
        m_pos++;
        int nargs = 0;
        skip();
        if (!accept(")")) {
          do { p_ternary(); nargs++; } while (accept(","));
          if (!accept(")")) fail("Missing parenthesis", name);
        }
        call(name, nargs);
        return;
      }
      auto v = m_vars.find(name);
      if (v != m_vars.end()) {
        Ins i = {VAR, 0, v->second, nullptr, nullptr, nullptr};
        m_prog.push_back(i);
        return;
      }
      double cval;
      auto c = m_consts.find(name);
      if (c != m_consts.end()) cval = c->second;
      else if (name == "_pi") cval = 3.141592653589793238462643;
      else if (name == "_e") cval = 2.718281828459045235360287;
      else fail("Unexpected token \"" + name + "\" found", name);
      Ins i = {PUSH, cval, nullptr, nullptr, nullptr, nullptr};
      m_prog.push_back(i);
      return;
    }
    fail("Unexpected token", std::string(1, ch));
  }

  void call(const std::string &name, int nargs) const {
    Ins i = {F1, 0, nullptr, nullptr, nullptr, nullptr};
    if (nargs == 1) {
      auto u = m_f1.find(name);
      if (u != m_f1.end()) { i.f1 = u->second; m_prog.push_back(i); return; }
      static const std::map<std::string, fun1_t> b1 = {
          {"sin", (fun1_t)std::sin},   {"cos", (fun1_t)std::cos},     {"tan", (fun1_t)std::tan},
          {"asin", (fun1_t)std::asin}, {"acos", (fun1_t)std::acos},   {"atan", (fun1_t)std::atan},
          {"sinh", (fun1_t)std::sinh}, {"cosh", (fun1_t)std::cosh},   {"tanh", (fun1_t)std::tanh},
          {"asinh", (fun1_t)std::asinh}, {"acosh", (fun1_t)std::acosh}, {"atanh", (fun1_t)std::atanh},
          {"exp", (fun1_t)std::exp},   {"log", b_log},                {"ln", b_log},
          {"log2", (fun1_t)std::log2}, {"log10", (fun1_t)std::log10}, {"sqrt", (fun1_t)std::sqrt},
          {"abs", (fun1_t)std::fabs},  {"sign", b_sign},              {"rint", b_rint}};
      auto b = b1.find(name);
      if (b != b1.end()) { i.f1 = b->second; m_prog.push_back(i); return; }
    } else if (nargs == 2) {
      i.op = F2;
      auto u = m_f2.find(name);
      if (u != m_f2.end()) { i.f2 = u->second; m_prog.push_back(i); return; }
      if (name == "min") { i.f2 = b_min; m_prog.push_back(i); return; }
      if (name == "max") { i.f2 = b_max; m_prog.push_back(i); return; }
    } else if (nargs == 3) {
      i.op = F3;
      auto u = m_f3.find(name);
      if (u != m_f3.end()) { i.f3 = u->second; m_prog.push_back(i); return; }
    }
    fail("Unknown function or wrong argument count", name);
  }

  std::string m_expr;
  std::map<std::string, double *> m_vars;
  std::map<std::string, double> m_consts;
  std::map<std::string, fun1_t> m_f1;
  std::map<std::string, fun2_t> m_f2;
  std::map<std::string, fun3_t> m_f3;
  mutable std::vector<Ins> m_prog;
  mutable size_t m_pos = 0;
  mutable bool m_dirty;
};

}  // namespace mu
#endif
