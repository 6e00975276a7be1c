// muParser.h (drop-in) -- mu::Parser, the expression evaluator ATUS-2
// programs use for potentials, initial states and AMP_T (rt_solver.cpp:
// 79-113, sob_solver.cpp:73-137, CRT_Base_IF.h:178-184), backed by the
// engine's own compiled evaluator (host/expr.h: muParser's grammar and
// precedence, the usual functions, user functions of one to three
// arguments).  Errors are thrown as mu::Parser::exception_type with
// GetMsg / GetExpr / GetToken / GetPos / GetCode, as the programs' catch
// blocks expect.  Not a general muParser replacement: no string variables,
// no bulk evaluation, no user operators.
#ifndef ATUS_DROPIN_MUPARSER_H
#define ATUS_DROPIN_MUPARSER_H

#include <iostream>
#include <string>

#include "../host/expr.h"

namespace mu {

typedef double value_type;
typedef std::string string_type;

class ParserError {
 public:
  ParserError(const std::string &msg, const std::string &expr, int pos, int code)
      : m_msg(msg), m_expr(expr), m_pos(pos), m_code(code) {}
  const std::string &GetMsg() const { return m_msg; }
  const std::string &GetExpr() const { return m_expr; }
  const std::string &GetToken() const { return m_token; }
  int GetPos() const { return m_pos; }
  int GetCode() const { return m_code; }

 private:
  std::string m_msg, m_expr, m_token;
  int m_pos, m_code;
};

class Parser {
 public:
  typedef ParserError exception_type;
  typedef double (*fun_type1)(double);
  typedef double (*fun_type2)(double, double);
  typedef double (*fun_type3)(double, double, double);

  void SetExpr(const std::string &e) { m_e.SetExpr(e); }
  const std::string &GetExpr() const { return m_e.GetExpr(); }
  void DefineVar(const std::string &name, double *p) { m_e.DefineVar(name, p); }
  void DefineConst(const std::string &name, double v) { m_e.DefineConst(name, v); }
  void DefineFun(const std::string &name, fun_type1 f, bool = true) { m_e.DefineFun(name, f); }
  void DefineFun(const std::string &name, fun_type2 f, bool = true) { m_e.DefineFun(name, f); }
  void DefineFun(const std::string &name, fun_type3 f, bool = true) { m_e.DefineFun(name, f); }
  void ClearConst() { m_e.ClearConst(); }
  double Eval() {
    try {
      return m_e.Eval();
    } catch (const atus::ExprError &err) {
      throw ParserError(err.what(), m_e.GetExpr(), (int)err.where, 1);
    }
  }

 private:
  atus::Expr m_e;
};

}  // namespace mu

#endif
