// expr.h -- run-time arithmetic expressions for the XML programs.
//
// The ATUS-2 programs read potentials, initial states and the pulse envelope
// as formulas in the XML file (POTENTIAL_xD, GUESS_xD, AMP_T) and evaluate
// them with muParser over the constants of the CONSTANTS section
// (ParameterHandler::Setup_muParser, ParameterHandler.cpp:298-312).  This is
// the engine's own evaluator for that role: a Pratt parser that compiles the
// text once into a postfix program of doubles, then evaluates it per point.
//
// Grammar (muParser's precedence): c ? a : b  <  ||  <  &&  <  comparisons
// <  + -  <  * /  <  unary + -  <  ^ (right associative), so -x^2 = -(x^2).
// Functions: sin cos tan asin acos atan sinh cosh tanh exp log ln log2 log10
// sqrt abs sign rint, min max (2 args), and user functions of 1..3 args;
// constants _pi and _e.  Errors throw atus::ExprError.
#pragma once

#include <cmath>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace atus {

struct ExprError : std::runtime_error {
  ExprError(const std::string &m, const std::string &expr, size_t pos)
      : std::runtime_error(m + " at position " + std::to_string(pos) + " in \"" + expr + "\""), where(pos) {}
  size_t where;
};

class Expr {
 public:
  using F1 = double (*)(double);
  using F2 = double (*)(double, double);
  using F3 = double (*)(double, double, double);

  Expr() = default;
  explicit Expr(const std::string &text) { SetExpr(text); }

  void SetExpr(const std::string &text) { src_ = text; compiled_ = false; }
  void DefineVar(const std::string &name, double *p) { vars_[name] = p; compiled_ = false; }
  void DefineConst(const std::string &name, double v) { consts_[name] = v; compiled_ = false; }
  void DefineFun(const std::string &name, F1 f) { fn_[name] = Fn{1, (void *)f}; compiled_ = false; }
  void DefineFun(const std::string &name, F2 f) { fn_[name] = Fn{2, (void *)f}; compiled_ = false; }
  void DefineFun(const std::string &name, F3 f) { fn_[name] = Fn{3, (void *)f}; compiled_ = false; }
  void ClearConst() { consts_.clear(); compiled_ = false; }
  const std::string &GetExpr() const { return src_; }

  double Eval() {
    if (!compiled_) compile();
    double st[64];
    int sp = -1;
    for (const Code &c : code_) {
      switch (c.op) {
        case NUM: st[++sp] = c.v; break;
        case VAR: st[++sp] = *c.p; break;
        case NEG: st[sp] = -st[sp]; break;
        case ADD: st[sp - 1] += st[sp]; sp--; break;
        case SUB: st[sp - 1] -= st[sp]; sp--; break;
        case MUL: st[sp - 1] *= st[sp]; sp--; break;
        case DIV: st[sp - 1] /= st[sp]; sp--; break;
        case POW: st[sp - 1] = std::pow(st[sp - 1], st[sp]); sp--; break;
        case LT: st[sp - 1] = st[sp - 1] < st[sp]; sp--; break;
        case LE: st[sp - 1] = st[sp - 1] <= st[sp]; sp--; break;
        case GT: st[sp - 1] = st[sp - 1] > st[sp]; sp--; break;
        case GE: st[sp - 1] = st[sp - 1] >= st[sp]; sp--; break;
        case EQ: st[sp - 1] = st[sp - 1] == st[sp]; sp--; break;
        case NE: st[sp - 1] = st[sp - 1] != st[sp]; sp--; break;
        case AND: st[sp - 1] = (st[sp - 1] != 0.0) && (st[sp] != 0.0); sp--; break;
        case OR: st[sp - 1] = (st[sp - 1] != 0.0) || (st[sp] != 0.0); sp--; break;
        case IF: st[sp - 2] = (st[sp - 2] != 0.0) ? st[sp - 1] : st[sp]; sp -= 2; break;
        case CALL1: st[sp] = ((F1)c.f)(st[sp]); break;
        case CALL2: st[sp - 1] = ((F2)c.f)(st[sp - 1], st[sp]); sp--; break;
        case CALL3: st[sp - 2] = ((F3)c.f)(st[sp - 2], st[sp - 1], st[sp]); sp -= 2; break;
      }
    }
    return st[0];
  }

 private:
  enum Op { NUM, VAR, NEG, ADD, SUB, MUL, DIV, POW, LT, LE, GT, GE, EQ, NE, AND, OR, IF, CALL1, CALL2, CALL3 };
  struct Code {
    Op op;
    double v = 0;
    const double *p = nullptr;
    void *f = nullptr;
  };
  struct Fn {
    int arity;
    void *f;
  };
  enum Tok { T_END, T_NUM, T_ID, T_OP, T_LP, T_RP, T_COMMA };

  // ---- lexer
  struct Token {
    Tok t;
    std::string s;
    double v = 0;
    size_t pos = 0;
  };
  Token next() {
    while (i_ < src_.size() && std::isspace((unsigned char)src_[i_])) i_++;
    Token tk;
    tk.pos = i_;
    if (i_ >= src_.size()) { tk.t = T_END; return tk; }
    const char ch = src_[i_];
    if (std::isdigit((unsigned char)ch) || (ch == '.' && i_ + 1 < src_.size() && std::isdigit((unsigned char)src_[i_ + 1]))) {
      char *end = nullptr;
      tk.v = std::strtod(src_.c_str() + i_, &end);
      i_ = (size_t)(end - src_.c_str());
      tk.t = T_NUM;
      return tk;
    }
    if (std::isalpha((unsigned char)ch) || ch == '_') {
      size_t j = i_;
      while (j < src_.size() && (std::isalnum((unsigned char)src_[j]) || src_[j] == '_')) j++;
      tk.t = T_ID;
      tk.s = src_.substr(i_, j - i_);
      i_ = j;
      return tk;
    }
    if (ch == '(') { i_++; tk.t = T_LP; return tk; }
    if (ch == ')') { i_++; tk.t = T_RP; return tk; }
    if (ch == ',') { i_++; tk.t = T_COMMA; return tk; }
    static const char *two[] = {"<=", ">=", "==", "!=", "&&", "||"};
    for (const char *op : two)
      if (src_.compare(i_, 2, op) == 0) { i_ += 2; tk.t = T_OP; tk.s = op; return tk; }
    if (std::string("+-*/^<>?:").find(ch) != std::string::npos) {
      i_++;
      tk.t = T_OP;
      tk.s = std::string(1, ch);
      return tk;
    }
    throw ExprError("unexpected character", src_, i_);
  }
  void advance() { cur_ = next(); }

  // binding powers: (left, right); right < left gives right associativity
  static int lbp(const std::string &op) {
    if (op == "?") return 1;
    if (op == "||") return 2;
    if (op == "&&") return 3;
    if (op == "<" || op == "<=" || op == ">" || op == ">=" || op == "==" || op == "!=") return 4;
    if (op == "+" || op == "-") return 5;
    if (op == "*" || op == "/") return 6;
    if (op == "^") return 8;
    return 0;
  }

  void emit(Op op) { Code c; c.op = op; code_.push_back(c); }

  void parse(int min_bp) {
    // prefix
    Token tk = cur_;
    if (tk.t == T_NUM) {
      advance();
      Code c; c.op = NUM; c.v = tk.v; code_.push_back(c);
    } else if (tk.t == T_ID) {
      advance();
      if (cur_.t == T_LP) {
        advance();
        int nargs = 0;
        if (cur_.t != T_RP) {
          for (;;) {
            parse(0);
            nargs++;
            if (cur_.t == T_COMMA) { advance(); continue; }
            break;
          }
        }
        if (cur_.t != T_RP) throw ExprError("missing ')'", src_, cur_.pos);
        advance();
        call(tk, nargs);
      } else {
        auto v = vars_.find(tk.s);
        if (v != vars_.end()) {
          Code c; c.op = VAR; c.p = v->second; code_.push_back(c);
        } else {
          double val;
          auto k = consts_.find(tk.s);
          if (k != consts_.end()) val = k->second;
          else if (tk.s == "_pi") val = 3.141592653589793238462643383279502884;
          else if (tk.s == "_e") val = 2.718281828459045235360287471352662498;
          else throw ExprError("unknown name \"" + tk.s + "\"", src_, tk.pos);
          Code c; c.op = NUM; c.v = val; code_.push_back(c);
        }
      }
    } else if (tk.t == T_LP) {
      advance();
      parse(0);
      if (cur_.t != T_RP) throw ExprError("missing ')'", src_, cur_.pos);
      advance();
    } else if (tk.t == T_OP && (tk.s == "-" || tk.s == "+")) {
      advance();
      parse(7);  // signs bind tighter than * / but looser than ^
      if (tk.s == "-") emit(NEG);
    } else {
      throw ExprError("unexpected token", src_, tk.pos);
    }
    // infix
    for (;;) {
      if (cur_.t != T_OP) return;
      const std::string op = cur_.s;
      const int bp = lbp(op);
      if (bp == 0 || bp <= min_bp) return;
      advance();
      if (op == "?") {
        parse(0);
        if (!(cur_.t == T_OP && cur_.s == ":")) throw ExprError("missing ':'", src_, cur_.pos);
        advance();
        parse(0);
        emit(IF);
        continue;
      }
      parse(op == "^" ? bp - 2 : bp);  // ^ right associative, its right side may carry a sign
      static const std::map<std::string, Op> ops = {{"+", ADD}, {"-", SUB}, {"*", MUL}, {"/", DIV}, {"^", POW},
                                                    {"<", LT},  {"<=", LE}, {">", GT},  {">=", GE}, {"==", EQ},
                                                    {"!=", NE}, {"&&", AND}, {"||", OR}};
      emit(ops.at(op));
    }
  }

  static double sgn(double x) { return (x > 0) - (x < 0); }
  static double mn(double a, double b) { return a < b ? a : b; }
  static double mx(double a, double b) { return a > b ? a : b; }

  void call(const Token &tk, int nargs) {
    Code c;
    auto u = fn_.find(tk.s);
    if (u != fn_.end()) {
      if (u->second.arity != nargs) throw ExprError("wrong argument count for " + tk.s, src_, tk.pos);
      c.op = nargs == 1 ? CALL1 : (nargs == 2 ? CALL2 : CALL3);
      c.f = u->second.f;
      code_.push_back(c);
      return;
    }
    static const std::map<std::string, F1> f1 = {
        {"sin", [](double x) { return std::sin(x); }},     {"cos", [](double x) { return std::cos(x); }},
        {"tan", [](double x) { return std::tan(x); }},     {"asin", [](double x) { return std::asin(x); }},
        {"acos", [](double x) { return std::acos(x); }},   {"atan", [](double x) { return std::atan(x); }},
        {"sinh", [](double x) { return std::sinh(x); }},   {"cosh", [](double x) { return std::cosh(x); }},
        {"tanh", [](double x) { return std::tanh(x); }},   {"exp", [](double x) { return std::exp(x); }},
        {"log", [](double x) { return std::log(x); }},     {"ln", [](double x) { return std::log(x); }},
        {"log2", [](double x) { return std::log2(x); }},   {"log10", [](double x) { return std::log10(x); }},
        {"sqrt", [](double x) { return std::sqrt(x); }},   {"abs", [](double x) { return std::fabs(x); }},
        {"sign", sgn},                                     {"rint", [](double x) { return std::rint(x); }}};
    if (nargs == 1) {
      auto f = f1.find(tk.s);
      if (f != f1.end()) { c.op = CALL1; c.f = (void *)f->second; code_.push_back(c); return; }
    }
    if (nargs == 2 && (tk.s == "min" || tk.s == "max")) {
      c.op = CALL2;
      c.f = (void *)(tk.s == "min" ? (F2)mn : (F2)mx);
      code_.push_back(c);
      return;
    }
    throw ExprError("unknown function " + tk.s, src_, tk.pos);
  }

  void compile() {
    code_.clear();
    i_ = 0;
    advance();
    if (cur_.t == T_END) throw ExprError("empty expression", src_, 0);
    parse(0);
    if (cur_.t != T_END) throw ExprError("unexpected trailing input", src_, cur_.pos);
    compiled_ = true;
  }

  std::string src_;
  std::map<std::string, double *> vars_;
  std::map<std::string, double> consts_;
  std::map<std::string, Fn> fn_;
  std::vector<Code> code_;
  Token cur_;
  size_t i_ = 0;
  bool compiled_ = false;
};

// Heaviside / rect / sign as ATUS-2 defines them (source/libs/lib_myutils/
// misc.cpp:40-53): sign = copysign(1, x), Heaviside = (1 + sign)/2 (so
// Heaviside(+0) = 1), rect(x, l, r) = Heaviside(x-l) - Heaviside(x-r).
inline double atus_sign(double x) { return std::copysign(1.0, x); }
inline double atus_heaviside(double x) { return 0.5 * (1.0 + atus_sign(x)); }
inline double atus_rect(double x, double l, double r) { return atus_heaviside(x - l) - atus_heaviside(x - r); }

}  // namespace atus
