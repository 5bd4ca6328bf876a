// opcount.hpp -- counting floating-point types for the op-count builds (test infrastructure).
//
// OpcF and OpcD have the size and layout of float and double and count every arithmetic operation
// done on them.  A C or C++ translation unit compiled with `#define float OpcF` / `#define double
// OpcD` after its system headers (see count_oracle.cc, count_emu.cc, count_eos.cc) then counts the
// operations its algorithm performs: the algorithmic work of the restatement, independent of the
// compiler and the GPU.
//
// Categories: add (+, -), mul (*), div (/), fma (fmaf / fma: 2 flops), sqrt (sqrt, cbrt), exp (exp,
// expf, pow of a non-integer, log, log10), trig (sin, cos, atan, acos).  flops = add + mul + div +
// 2 fma; the special functions are reported separately (the GPU evaluates them on its SFU or by
// library sequences).  Comparisons, conversions and copies are not counted.
#pragma once

#include <math.h>

namespace opc {

struct Counts {
  long long add = 0, mul = 0, div = 0, fma = 0, sqrt = 0, exp = 0, trig = 0;
  long long flops() const { return add + mul + div + 2 * fma; }
  void reset() { *this = Counts(); }
};

extern Counts c32, c64;  // operations on OpcF and on OpcD (mixed ones count as OpcD)

}  // namespace opc

struct OpcD;

struct OpcF {
  float v;
  OpcF() = default;
  constexpr OpcF(float x) : v(x) {}
  constexpr OpcF(double x) : v((float)x) {}
  constexpr OpcF(int x) : v((float)x) {}
  constexpr OpcF(long x) : v((float)x) {}
  constexpr OpcF(unsigned x) : v((float)x) {}
  constexpr OpcF(long long x) : v((float)x) {}
  constexpr OpcF(unsigned long x) : v((float)x) {}
  constexpr OpcF(const OpcD &d);
  explicit operator float() const { return v; }
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  explicit operator long() const { return (long)v; }
  explicit operator bool() const { return v != 0.f; }
};

struct OpcD {
  double v;
  OpcD() = default;
  constexpr OpcD(double x) : v(x) {}
  constexpr OpcD(float x) : v(x) {}
  constexpr OpcD(int x) : v(x) {}
  constexpr OpcD(long x) : v((double)x) {}
  constexpr OpcD(unsigned x) : v(x) {}
  constexpr OpcD(long long x) : v((double)x) {}
  constexpr OpcD(unsigned long x) : v((double)x) {}
  constexpr OpcD(const OpcF &f) : v(f.v) {}
  explicit operator double() const { return v; }
  explicit operator float() const { return (float)v; }
  explicit operator int() const { return (int)v; }
  explicit operator long() const { return (long)v; }
  explicit operator bool() const { return v != 0.0; }
};

constexpr OpcF::OpcF(const OpcD &d) : v((float)d.v) {}

// ---- arithmetic: OpcF op OpcF -> OpcF; anything with OpcD or a double literal -> OpcD ------------
#define OPC_BIN(OP, CAT)                                                                             \
  inline OpcF operator OP(OpcF a, OpcF b) { ++opc::c32.CAT; return OpcF(a.v OP b.v); }              \
  inline OpcF operator OP(OpcF a, float b) { ++opc::c32.CAT; return OpcF(a.v OP b); }               \
  inline OpcF operator OP(float a, OpcF b) { ++opc::c32.CAT; return OpcF(a OP b.v); }               \
  inline OpcF operator OP(OpcF a, int b) { ++opc::c32.CAT; return OpcF(a.v OP (float)b); }          \
  inline OpcF operator OP(int a, OpcF b) { ++opc::c32.CAT; return OpcF((float)a OP b.v); }          \
  inline OpcD operator OP(OpcF a, double b) { ++opc::c64.CAT; return OpcD((double)a.v OP b); }      \
  inline OpcD operator OP(double a, OpcF b) { ++opc::c64.CAT; return OpcD(a OP (double)b.v); }      \
  inline OpcD operator OP(OpcD a, OpcD b) { ++opc::c64.CAT; return OpcD(a.v OP b.v); }              \
  inline OpcD operator OP(OpcD a, double b) { ++opc::c64.CAT; return OpcD(a.v OP b); }              \
  inline OpcD operator OP(double a, OpcD b) { ++opc::c64.CAT; return OpcD(a OP b.v); }              \
  inline OpcD operator OP(OpcD a, float b) { ++opc::c64.CAT; return OpcD(a.v OP (double)b); }       \
  inline OpcD operator OP(float a, OpcD b) { ++opc::c64.CAT; return OpcD((double)a OP b.v); }       \
  inline OpcD operator OP(OpcD a, int b) { ++opc::c64.CAT; return OpcD(a.v OP (double)b); }         \
  inline OpcD operator OP(int a, OpcD b) { ++opc::c64.CAT; return OpcD((double)a OP b.v); }         \
  inline OpcD operator OP(OpcD a, long b) { ++opc::c64.CAT; return OpcD(a.v OP (double)b); }        \
  inline OpcD operator OP(long a, OpcD b) { ++opc::c64.CAT; return OpcD((double)a OP b.v); }        \
  inline OpcD operator OP(OpcD a, OpcF b) { ++opc::c64.CAT; return OpcD(a.v OP (double)b.v); }      \
  inline OpcD operator OP(OpcF a, OpcD b) { ++opc::c64.CAT; return OpcD((double)a.v OP b.v); }
OPC_BIN(+, add)
OPC_BIN(-, add)
OPC_BIN(*, mul)
OPC_BIN(/, div)
#undef OPC_BIN

#define OPC_ASSIGN(OP, BOP)                                                                        \
  template <typename T> inline OpcF &operator OP(OpcF &a, const T &b) { a = a BOP b; return a; }  \
  template <typename T> inline OpcD &operator OP(OpcD &a, const T &b) { a = a BOP b; return a; }
OPC_ASSIGN(+=, +)
OPC_ASSIGN(-=, -)
OPC_ASSIGN(*=, *)
OPC_ASSIGN(/=, /)
#undef OPC_ASSIGN

inline OpcF operator-(OpcF a) { return OpcF(-a.v); }
inline OpcD operator-(OpcD a) { return OpcD(-a.v); }
inline OpcF operator+(OpcF a) { return a; }
inline OpcD operator+(OpcD a) { return a; }

// ---- comparisons (not counted) -------------------------------------------------------------------
#define OPC_CMP(OP)                                                          \
  inline bool operator OP(OpcF a, OpcF b) { return a.v OP b.v; }             \
  inline bool operator OP(OpcF a, float b) { return a.v OP b; }              \
  inline bool operator OP(float a, OpcF b) { return a OP b.v; }              \
  inline bool operator OP(OpcF a, double b) { return a.v OP b; }             \
  inline bool operator OP(double a, OpcF b) { return a OP b.v; }             \
  inline bool operator OP(OpcF a, int b) { return a.v OP b; }                \
  inline bool operator OP(int a, OpcF b) { return a OP b.v; }                \
  inline bool operator OP(OpcD a, OpcD b) { return a.v OP b.v; }             \
  inline bool operator OP(OpcD a, double b) { return a.v OP b; }             \
  inline bool operator OP(double a, OpcD b) { return a OP b.v; }             \
  inline bool operator OP(OpcD a, float b) { return a.v OP b; }              \
  inline bool operator OP(float a, OpcD b) { return a OP b.v; }              \
  inline bool operator OP(OpcD a, int b) { return a.v OP b; }                \
  inline bool operator OP(int a, OpcD b) { return a OP b.v; }                \
  inline bool operator OP(OpcD a, OpcF b) { return a.v OP b.v; }             \
  inline bool operator OP(OpcF a, OpcD b) { return a.v OP b.v; }
OPC_CMP(<)
OPC_CMP(>)
OPC_CMP(<=)
OPC_CMP(>=)
OPC_CMP(==)
OPC_CMP(!=)
#undef OPC_CMP

// ---- math functions --------------------------------------------------------------------------------
inline OpcF sqrtf(OpcF a) { ++opc::c32.sqrt; return OpcF(::sqrtf(a.v)); }
inline OpcF expf(OpcF a) { ++opc::c32.exp; return OpcF(::expf(a.v)); }
inline OpcF logf(OpcF a) { ++opc::c32.exp; return OpcF(::logf(a.v)); }
inline OpcF log10f(OpcF a) { ++opc::c32.exp; return OpcF(::log10f(a.v)); }
inline OpcF sinf(OpcF a) { ++opc::c32.trig; return OpcF(::sinf(a.v)); }
inline OpcF cosf(OpcF a) { ++opc::c32.trig; return OpcF(::cosf(a.v)); }
inline OpcF fabsf(OpcF a) { return OpcF(::fabsf(a.v)); }
inline OpcF fminf(OpcF a, OpcF b) { return OpcF(::fminf(a.v, b.v)); }
inline OpcF fmaxf(OpcF a, OpcF b) { return OpcF(::fmaxf(a.v, b.v)); }
inline OpcF floorf(OpcF a) { return OpcF(::floorf(a.v)); }
inline OpcF copysignf(OpcF a, OpcF b) { return OpcF(::copysignf(a.v, b.v)); }
inline OpcF fmaf(OpcF a, OpcF b, OpcF c) { ++opc::c32.fma; return OpcF(::fmaf(a.v, b.v, c.v)); }
inline OpcF powf(OpcF a, OpcF b) { ++opc::c32.exp; return OpcF(::powf(a.v, b.v)); }
inline bool isfinite(OpcF a) { return ::isfinite(a.v); }
inline bool isnan(OpcF a) { return ::isnan(a.v); }

inline OpcD sqrt(OpcD a) { ++opc::c64.sqrt; return OpcD(::sqrt(a.v)); }
inline OpcD cbrt(OpcD a) { ++opc::c64.sqrt; return OpcD(::cbrt(a.v)); }
inline OpcD exp(OpcD a) { ++opc::c64.exp; return OpcD(::exp(a.v)); }
inline OpcD log(OpcD a) { ++opc::c64.exp; return OpcD(::log(a.v)); }
inline OpcD log10(OpcD a) { ++opc::c64.exp; return OpcD(::log10(a.v)); }
inline OpcD sin(OpcD a) { ++opc::c64.trig; return OpcD(::sin(a.v)); }
inline OpcD cos(OpcD a) { ++opc::c64.trig; return OpcD(::cos(a.v)); }
inline OpcD atan(OpcD a) { ++opc::c64.trig; return OpcD(::atan(a.v)); }
inline OpcD acos(OpcD a) { ++opc::c64.trig; return OpcD(::acos(a.v)); }
inline OpcD fabs(OpcD a) { return OpcD(::fabs(a.v)); }
inline OpcD fmin(OpcD a, OpcD b) { return OpcD(::fmin(a.v, b.v)); }
inline OpcD fmax(OpcD a, OpcD b) { return OpcD(::fmax(a.v, b.v)); }
inline OpcD floor(OpcD a) { return OpcD(::floor(a.v)); }
inline OpcD fma(OpcD a, OpcD b, OpcD c) { ++opc::c64.fma; return OpcD(::fma(a.v, b.v, c.v)); }
// pow: an integer power is repeated multiplication (what a compiler emits), else exp / log
inline OpcD pow(OpcD a, int n) {
  double r = 1.0;
  for (int i = 0; i < (n < 0 ? -n : n); ++i) { r *= a.v; if (i) ++opc::c64.mul; }
  if (n < 0) { ++opc::c64.div; r = 1.0 / r; }
  return OpcD(r);
}
inline OpcD pow(OpcD a, OpcD b) {
  if (b.v == (double)(int)b.v && b.v >= -8 && b.v <= 8) return pow(a, (int)b.v);
  ++opc::c64.exp;
  return OpcD(::pow(a.v, b.v));
}
inline OpcD pow(OpcD a, double b) { return pow(a, OpcD(b)); }
inline OpcD pow(double a, OpcD b) { return pow(OpcD(a), b); }
inline bool isfinite(OpcD a) { return ::isfinite(a.v); }
inline bool isnan(OpcD a) { return ::isnan(a.v); }
