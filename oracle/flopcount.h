/* flopcount.h -- counting FP64 scalar for the oracle (test infrastructure).
 * Compiling oracle/nr_oracle.c as C++ with -DORACLE_COUNT_FLOPS replaces its
 * scalar type by fcdouble, which counts + - * / (1 FLOP each) and the
 * transcendental calls log/exp/pow (separately).  Comparisons are free. */
#pragma once
#include <cmath>
struct fc_counts { long long flops, transc; };
extern fc_counts g_fc;
struct fcdouble {
  double v;
  fcdouble() : v(0) {}
  fcdouble(double x) : v(x) {}
  fcdouble &operator+=(const fcdouble &o) { g_fc.flops++; v += o.v; return *this; }
  fcdouble &operator-=(const fcdouble &o) { g_fc.flops++; v -= o.v; return *this; }
  fcdouble &operator*=(const fcdouble &o) { g_fc.flops++; v *= o.v; return *this; }
  fcdouble operator-() const { return fcdouble(-v); }
};
#define FC_BIN(op)                                                                               \
  inline fcdouble operator op(const fcdouble &a, const fcdouble &b) { g_fc.flops++; return fcdouble(a.v op b.v); } \
  inline fcdouble operator op(const fcdouble &a, double b) { g_fc.flops++; return fcdouble(a.v op b); }           \
  inline fcdouble operator op(double a, const fcdouble &b) { g_fc.flops++; return fcdouble(a op b.v); }
FC_BIN(+) FC_BIN(-) FC_BIN(*) FC_BIN(/)
#undef FC_BIN
#define FC_CMP(op)                                                                   \
  inline bool operator op(const fcdouble &a, const fcdouble &b) { return a.v op b.v; } \
  inline bool operator op(const fcdouble &a, double b) { return a.v op b; }
FC_CMP(<) FC_CMP(>) FC_CMP(<=) FC_CMP(>=) FC_CMP(==) FC_CMP(!=)
#undef FC_CMP
inline fcdouble fc_log(const fcdouble &a) { g_fc.transc++; return fcdouble(std::log(a.v)); }
inline fcdouble fc_exp(const fcdouble &a) { g_fc.transc++; return fcdouble(std::exp(a.v)); }
inline fcdouble fc_pow(const fcdouble &a, double b) { g_fc.transc++; return fcdouble(std::pow(a.v, b)); }
inline double fc_val(const fcdouble &a) { return a.v; }
