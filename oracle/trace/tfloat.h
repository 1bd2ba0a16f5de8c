// A float stand-in that records every comparison it takes part in
// (test infrastructure: the cut-flip tracer and the FP64 re-evaluation of
// oracle/trace/lst_trace.cc).
//
// The tracer compiles the product's cut headers (tracklooper_b200/csrc/
// lst_*.h, written for float) with `float` defined as TFloat.  A TFloat holds
// a double and runs in one of three modes, chosen per evaluation:
//
//   kF32Cr     every float operation rounds to float, exactly as IEEE single
//              precision does (+ - * / and sqrt are computed in double and
//              rounded once, which is exact for these operations because a
//              double carries more than 2 x 24 + 2 bits); transcendentals
//              are float(f(double(x))), the binding of the CUDA path and of
//              the parity oracle;
//   kF32Glibc  as kF32Cr, with glibc's float transcendentals (sinf,
//              atan2f, ...), the binding of the reference's stock CPU build;
//   kF64       nothing is rounded to float: the same formulas evaluated in
//              double precision from the same float inputs.
//
// C++ promotes float to double where an expression mixes the two; TFloat
// mixed with double therefore yields a plain double, and TFloat mixed with an
// integer yields a TFloat, as float does.  Constants that the headers declare
// constexpr float are rounded to float in every mode (they are float
// constants of the reference).
//
// Every comparison with a TFloat operand appends (site, lhs, rhs, op,
// result) to the current thread's trace, site being the code address of the
// comparison (resolved to file:line by the tracer's Python side).
#pragma once

#include <cmath>
#include <cstdint>
#include <type_traits>
#include <vector>

namespace lst_trace {

  enum Mode : int { kF32Cr = 0, kF32Glibc = 1, kF64 = 2 };
  enum CmpOp : int { kLT = 0, kLE = 1, kGT = 2, kGE = 3, kEQ = 4, kNE = 5 };

  struct Rec {
    const void* site;
    double lhs, rhs;
    int op;
    int result;
  };

  inline thread_local int g_mode = kF32Cr;
  inline thread_local std::vector<Rec>* g_trace = nullptr;

  // Rounds a result as the current mode does; in a constant expression (a
  // constexpr float of the headers) always to float.
  constexpr double rnd(double v) {
    if (std::is_constant_evaluated())
      return static_cast<double>(static_cast<float>(v));
    return g_mode == kF64 ? v : static_cast<double>(static_cast<float>(v));
  }

  // Appends one comparison to the current trace (if one is being recorded).
  __attribute__((noinline)) inline void record(const void* site, double a, double b, int op, bool r) {
    if (g_trace)
      g_trace->push_back(Rec{site, a, b, op, r ? 1 : 0});
  }

#define LST_TRACE_SITE __builtin_extract_return_addr(__builtin_return_address(0))

  struct TFloat {
    double v;
    constexpr TFloat() : v(0) {}
    constexpr TFloat(float f) : v(f) {}
    constexpr TFloat(double d) : v(rnd(d)) {}
    template <typename I, typename = std::enable_if_t<std::is_integral_v<I>>>
    constexpr TFloat(I i) : TFloat(static_cast<double>(i)) {}
    explicit constexpr operator double() const { return v; }
    template <typename I, typename = std::enable_if_t<std::is_integral_v<I>>>
    explicit constexpr operator I() const {
      return static_cast<I>(v);
    }
    constexpr TFloat operator-() const { return TFloat::raw(-v); }
    constexpr TFloat operator+() const { return *this; }
    static constexpr TFloat raw(double d) {
      TFloat t;
      t.v = d;
      return t;
    }
    TFloat& operator+=(TFloat o) { v = rnd(v + o.v); return *this; }
    TFloat& operator-=(TFloat o) { v = rnd(v - o.v); return *this; }
    TFloat& operator*=(TFloat o) { v = rnd(v * o.v); return *this; }
    TFloat& operator/=(TFloat o) { v = rnd(v / o.v); return *this; }
    TFloat& operator+=(double o) { v = rnd(v + o); return *this; }
    TFloat& operator-=(double o) { v = rnd(v - o); return *this; }
    TFloat& operator*=(double o) { v = rnd(v * o); return *this; }
    TFloat& operator/=(double o) { v = rnd(v / o); return *this; }
  };

  template <typename T>
  constexpr bool kIsInt = std::is_integral_v<T>;

  // TFloat (op) TFloat -> TFloat
  constexpr TFloat operator+(TFloat a, TFloat b) { return TFloat::raw(rnd(a.v + b.v)); }
  constexpr TFloat operator-(TFloat a, TFloat b) { return TFloat::raw(rnd(a.v - b.v)); }
  constexpr TFloat operator*(TFloat a, TFloat b) { return TFloat::raw(rnd(a.v * b.v)); }
  constexpr TFloat operator/(TFloat a, TFloat b) { return TFloat::raw(rnd(a.v / b.v)); }
  // TFloat (op) float literal -> TFloat
  constexpr TFloat operator+(TFloat a, float b) { return a + TFloat(b); }
  constexpr TFloat operator-(TFloat a, float b) { return a - TFloat(b); }
  constexpr TFloat operator*(TFloat a, float b) { return a * TFloat(b); }
  constexpr TFloat operator/(TFloat a, float b) { return a / TFloat(b); }
  constexpr TFloat operator+(float a, TFloat b) { return TFloat(a) + b; }
  constexpr TFloat operator-(float a, TFloat b) { return TFloat(a) - b; }
  constexpr TFloat operator*(float a, TFloat b) { return TFloat(a) * b; }
  constexpr TFloat operator/(float a, TFloat b) { return TFloat(a) / b; }
  // TFloat (op) double -> double (C++ promotes the float)
  constexpr double operator+(TFloat a, double b) { return a.v + b; }
  constexpr double operator-(TFloat a, double b) { return a.v - b; }
  constexpr double operator*(TFloat a, double b) { return a.v * b; }
  constexpr double operator/(TFloat a, double b) { return a.v / b; }
  constexpr double operator+(double a, TFloat b) { return a + b.v; }
  constexpr double operator-(double a, TFloat b) { return a - b.v; }
  constexpr double operator*(double a, TFloat b) { return a * b.v; }
  constexpr double operator/(double a, TFloat b) { return a / b.v; }
  // TFloat (op) integer -> TFloat (the integer converts to float)
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator+(TFloat a, I b) { return a + TFloat(b); }
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator-(TFloat a, I b) { return a - TFloat(b); }
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator*(TFloat a, I b) { return a * TFloat(b); }
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator/(TFloat a, I b) { return a / TFloat(b); }
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator+(I a, TFloat b) { return TFloat(a) + b; }
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator-(I a, TFloat b) { return TFloat(a) - b; }
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator*(I a, TFloat b) { return TFloat(a) * b; }
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>
  constexpr TFloat operator/(I a, TFloat b) { return TFloat(a) / b; }

  // Comparisons: recorded.  Each is out of line and records its own return
  // address, i.e. the instruction in the cut code right after the call.
#define LST_TRACE_CMP(OPSYM, OPCODE)                                                             \
  __attribute__((noinline)) inline bool operator OPSYM(TFloat a, TFloat b) {                    \
    bool r = a.v OPSYM b.v;                                                                      \
    record(LST_TRACE_SITE, a.v, b.v, OPCODE, r);                                                 \
    return r;                                                                                    \
  }                                                                                              \
  __attribute__((noinline)) inline bool operator OPSYM(TFloat a, double b) {                    \
    bool r = a.v OPSYM b;                                                                        \
    record(LST_TRACE_SITE, a.v, b, OPCODE, r);                                                   \
    return r;                                                                                    \
  }                                                                                              \
  __attribute__((noinline)) inline bool operator OPSYM(double a, TFloat b) {                    \
    bool r = a OPSYM b.v;                                                                        \
    record(LST_TRACE_SITE, a, b.v, OPCODE, r);                                                   \
    return r;                                                                                    \
  }                                                                                              \
  __attribute__((noinline)) inline bool operator OPSYM(TFloat a, float b) {                     \
    bool r = a.v OPSYM static_cast<double>(b);                                                   \
    record(LST_TRACE_SITE, a.v, b, OPCODE, r);                                                   \
    return r;                                                                                    \
  }                                                                                              \
  __attribute__((noinline)) inline bool operator OPSYM(float a, TFloat b) {                     \
    bool r = static_cast<double>(a) OPSYM b.v;                                                   \
    record(LST_TRACE_SITE, a, b.v, OPCODE, r);                                                   \
    return r;                                                                                    \
  }                                                                                              \
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>                                  \
  __attribute__((noinline)) inline bool operator OPSYM(TFloat a, I b) {                         \
    double bb = TFloat(b).v;                                                                     \
    bool r = a.v OPSYM bb;                                                                       \
    record(LST_TRACE_SITE, a.v, bb, OPCODE, r);                                                  \
    return r;                                                                                    \
  }                                                                                              \
  template <typename I, typename = std::enable_if_t<kIsInt<I>>>                                  \
  __attribute__((noinline)) inline bool operator OPSYM(I a, TFloat b) {                         \
    double aa = TFloat(a).v;                                                                     \
    bool r = aa OPSYM b.v;                                                                       \
    record(LST_TRACE_SITE, aa, b.v, OPCODE, r);                                                  \
    return r;                                                                                    \
  }
  LST_TRACE_CMP(<, kLT)
  LST_TRACE_CMP(<=, kLE)
  LST_TRACE_CMP(>, kGT)
  LST_TRACE_CMP(>=, kGE)
  LST_TRACE_CMP(==, kEQ)
  LST_TRACE_CMP(!=, kNE)
#undef LST_TRACE_CMP

}  // namespace lst_trace
