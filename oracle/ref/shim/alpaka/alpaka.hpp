// Minimal serial stand-in for the subset of the Alpaka 1.1 API that the LST
// reference sources use (SDL/*.h, SDL/*.cc).  Test infrastructure only: it
// exists so that g++ can compile the unmodified reference CPU backend
// ("ALPAKA_ACC_CPU_B_SEQ_T_SEQ_ENABLED": one block, one thread, loops run in
// ascending index order) as the parity oracle.  Nothing in the product links it.
//
// Semantics reproduced:
//   * every work division collapses to 1x1x1 (SDL/Constants.h:88-92), so the
//     grid-stride loops of every kernel run serially in index order;
//   * atomics are plain read-modify-write (single thread);
//   * alpaka::math::* forwards to <cmath>.  Two bindings exist for the float
//     transcendentals, selected at compile time:
//       LSTREF_MATH_CR (default): float f(x) = (float) f((double) x), the
//         binding the CUDA product uses, so both sides round the same double;
//       LSTREF_MATH_NATIVE: float f(x) = std::f(float), i.e. glibc's float
//         functions, exactly what Alpaka's StdLib backend calls.
//     sqrt/abs/min/max/round/isnan are exact in both bindings.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#define ALPAKA_FN_ACC
#define ALPAKA_FN_HOST
#define ALPAKA_FN_HOST_ACC
#define ALPAKA_FN_INLINE inline
#define ALPAKA_STATIC_ACC_MEM_GLOBAL static

namespace alpaka {

  template <std::size_t N>
  using DimInt = std::integral_constant<std::size_t, N>;

  template <typename TDim, typename TVal>
  struct Vec {
    static constexpr std::size_t kDim = TDim::value;
    TVal v[kDim];
    Vec() : v{} {}
    template <typename... Ts, typename = std::enable_if_t<sizeof...(Ts) == kDim>>
    Vec(Ts... ts) : v{static_cast<TVal>(ts)...} {}
    static Vec all(TVal x) {
      Vec r;
      for (std::size_t i = 0; i < kDim; ++i)
        r.v[i] = x;
      return r;
    }
    TVal& operator[](std::size_t i) { return v[i]; }
    TVal const& operator[](std::size_t i) const { return v[i]; }
  };

  template <typename TDim, typename TIdx>
  struct WorkDivMembers {
    Vec<TDim, TIdx> blocks, threads, elems;
    WorkDivMembers(Vec<TDim, TIdx> const& b, Vec<TDim, TIdx> const& t, Vec<TDim, TIdx> const& e)
        : blocks(b), threads(t), elems(e) {}
  };

  // Index origins / units.
  struct Grid {};
  struct Block {};
  struct Threads {};
  struct Blocks {};

  // The serial accelerator: one block, one thread.
  template <typename TDim, typename TIdx>
  struct AccCpuSerial {};

  template <typename TOrigin, typename TUnit, typename TAcc>
  inline Vec<DimInt<3>, uint32_t> getIdx(TAcc const&) {
    return Vec<DimInt<3>, uint32_t>::all(0u);
  }
  template <typename TOrigin, typename TUnit, typename TAcc>
  inline Vec<DimInt<3>, uint32_t> getWorkDiv(TAcc const&) {
    return Vec<DimInt<3>, uint32_t>::all(1u);
  }

  // Devices, platform, queue.
  struct DevCpu {};
  struct PlatformCpu {};
  struct QueueCpuBlocking {
    DevCpu dev;
    QueueCpuBlocking() = default;
    explicit QueueCpuBlocking(DevCpu const& d) : dev(d) {}
  };
  template <typename T>
  using Dev = DevCpu;
  inline DevCpu getDev(QueueCpuBlocking const& q) { return q.dev; }
  inline DevCpu getDevByIdx(PlatformCpu const&, std::size_t) { return DevCpu{}; }
  inline void wait(QueueCpuBlocking const&) {}

  // Owning 1-D buffer with shared ownership (Alpaka buffers are reference counted).
  template <typename TDev, typename T, typename TDim, typename TIdx>
  class Buf {
  public:
    Buf() = default;
    explicit Buf(std::size_t n) : n_(n), p_(n ? new T[n] : nullptr, [](T* q) { delete[] q; }) {
      if (n)
        std::memset(static_cast<void*>(p_.get()), 0, n * sizeof(T));
    }
    T* data() const { return p_.get(); }
    std::size_t size() const { return n_; }

  private:
    std::size_t n_ = 0;
    std::shared_ptr<T> p_;
  };

  // Non-owning 1-D view (createView / createSubView).
  template <typename T>
  struct View {
    T* p;
    std::size_t n;
    T* data() const { return p; }
    std::size_t size() const { return n; }
  };

  namespace detail {
    template <typename E>
    inline std::size_t extentOf(E const& e) {
      if constexpr (std::is_integral_v<E>)
        return static_cast<std::size_t>(e);
      else
        return static_cast<std::size_t>(e[0]);
    }
    template <typename X>
    inline auto ptrOf(X& x) {
      return x.data();
    }
    template <typename X>
    inline auto ptrOf(X const& x) {
      return x.data();
    }
  }  // namespace detail

  template <typename T, typename TIdx, typename TDev, typename TExt>
  inline Buf<TDev, T, DimInt<1>, TIdx> allocBuf(TDev const&, TExt const& ext) {
    return Buf<TDev, T, DimInt<1>, TIdx>(detail::extentOf(ext));
  }

  template <typename TDev, typename T, typename TDim, typename TIdx>
  inline T* getPtrNative(Buf<TDev, T, TDim, TIdx> const& b) {
    return b.data();
  }

  template <typename TDev, typename T, typename TExt>
  inline View<T> createView(TDev const&, T* p, TExt const& ext) {
    return View<T>{p, detail::extentOf(ext)};
  }

  template <typename TDev, typename T, typename TDim, typename TIdx, typename TExt, typename TOff>
  inline View<T> createSubView(Buf<TDev, T, TDim, TIdx>& b, TExt const& ext, TOff const& off) {
    return View<T>{b.data() + detail::extentOf(off), detail::extentOf(ext)};
  }

  // memcpy between any two of {Buf, View, std::vector}; without an explicit
  // extent the smaller of the two sizes is copied.
  template <typename TQueue, typename TDst, typename TSrc, typename TExt>
  inline void memcpy(TQueue&, TDst&& dst, TSrc const& src, TExt const& ext) {
    std::size_t n = detail::extentOf(ext);
    if (n)
      std::memmove(static_cast<void*>(detail::ptrOf(dst)),
                   static_cast<void const*>(detail::ptrOf(src)),
                   n * sizeof(*detail::ptrOf(src)));
  }
  template <typename TQueue, typename TDst, typename TSrc>
  inline void memcpy(TQueue& q, TDst&& dst, TSrc const& src) {
    std::size_t n = std::min<std::size_t>(dst.size(), src.size());
    memcpy(q, dst, src, n);
  }

  template <typename TQueue, typename TView, typename TVal>
  inline void memset(TQueue&, TView& v, TVal const& val) {
    if (v.size())
      std::memset(static_cast<void*>(v.data()), static_cast<int>(val), v.size() * sizeof(*v.data()));
  }

  // Kernel launch: the task holds the functor and its arguments by value and
  // runs serially on enqueue.
  template <typename TAcc, typename TKernel, typename... TArgs>
  struct TaskKernel {
    TKernel kernel;
    std::tuple<std::decay_t<TArgs>...> args;
    void operator()() const {
      TAcc acc{};
      std::apply([&](auto const&... a) { kernel(acc, a...); }, args);
    }
  };
  template <typename TAcc, typename TWorkDiv, typename TKernel, typename... TArgs>
  inline TaskKernel<TAcc, TKernel, TArgs...> createTaskKernel(TWorkDiv const&, TKernel const& k, TArgs&&... a) {
    return TaskKernel<TAcc, TKernel, TArgs...>{k, std::tuple<std::decay_t<TArgs>...>(std::forward<TArgs>(a)...)};
  }
  template <typename TQueue, typename TTask>
  inline void enqueue(TQueue&, TTask const& t) {
    t();
  }

  // Atomics (single thread: plain read-modify-write, returning the old value).
  struct AtomicAdd {};
  struct AtomicSub {};
  struct AtomicMin {};
  struct AtomicMax {};
  struct AtomicCas {};
  template <typename TOp, typename TAcc, typename T, typename U>
  inline T atomicOp(TAcc const&, T* addr, U const& val) {
    T old = *addr;
    if constexpr (std::is_same_v<TOp, AtomicAdd>)
      *addr = static_cast<T>(old + val);
    else if constexpr (std::is_same_v<TOp, AtomicSub>)
      *addr = static_cast<T>(old - val);
    else if constexpr (std::is_same_v<TOp, AtomicMin>)
      *addr = (static_cast<T>(val) < old) ? static_cast<T>(val) : old;
    else if constexpr (std::is_same_v<TOp, AtomicMax>)
      *addr = (static_cast<T>(val) > old) ? static_cast<T>(val) : old;
    else
      static_assert(!sizeof(TOp), "unsupported atomic");
    return old;
  }
  template <typename TOp, typename TAcc, typename T, typename U, typename V>
  inline T atomicOp(TAcc const&, T* addr, U const& compare, V const& val) {
    static_assert(std::is_same_v<TOp, AtomicCas>, "4-argument atomicOp is compare-and-swap");
    T old = *addr;
    if (old == static_cast<T>(compare))
      *addr = static_cast<T>(val);
    return old;
  }

  // Block-shared variables: one instance per (type, id) and host thread, so
  // that events processed concurrently on different threads do not share them.
  template <typename T, std::size_t TUniqueId, typename TAcc>
  inline T& declareSharedVar(TAcc const&) {
    static thread_local T v;
    return v;
  }
  template <typename TAcc>
  inline void syncBlockThreads(TAcc const&) {}

  namespace math {
    template <typename TAcc, typename T>
    inline auto abs(TAcc const&, T const& x) {
      return std::abs(x);
    }
    template <typename TAcc, typename T>
    inline auto sqrt(TAcc const&, T const& x) {
      return std::sqrt(x);
    }
    template <typename TAcc, typename Tx, typename Ty>
    inline auto min(TAcc const&, Tx const& x, Ty const& y) {
      if constexpr (std::is_integral_v<Tx> && std::is_integral_v<Ty>)
        return std::min(x, y);
      else
        return std::fmin(x, y);
    }
    template <typename TAcc, typename Tx, typename Ty>
    inline auto max(TAcc const&, Tx const& x, Ty const& y) {
      if constexpr (std::is_integral_v<Tx> && std::is_integral_v<Ty>)
        return std::max(x, y);
      else
        return std::fmax(x, y);
    }
    template <typename TAcc, typename T>
    inline auto round(TAcc const&, T const& x) {
      return std::round(x);
    }
    template <typename TAcc, typename T>
    inline bool isnan(TAcc const&, T const& x) {
      return std::isnan(x);
    }

#if defined(LSTREF_MATH_NATIVE)
#define LSTREF_UNARY(name)                       \
  template <typename TAcc, typename T>           \
  inline auto name(TAcc const&, T const& x) {    \
    return std::name(x);                         \
  }
    template <typename TAcc, typename Ty, typename Tx>
    inline auto atan2(TAcc const&, Ty const& y, Tx const& x) {
      return std::atan2(y, x);
    }
#else
#define LSTREF_UNARY(name)                                      \
  template <typename TAcc, typename T>                          \
  inline auto name(TAcc const&, T const& x) {                   \
    if constexpr (std::is_same_v<T, float>)                     \
      return static_cast<float>(std::name(static_cast<double>(x))); \
    else                                                        \
      return std::name(x);                                      \
  }
    template <typename TAcc, typename Ty, typename Tx>
    inline auto atan2(TAcc const&, Ty const& y, Tx const& x) {
      if constexpr (std::is_same_v<Ty, float> && std::is_same_v<Tx, float>)
        return static_cast<float>(std::atan2(static_cast<double>(y), static_cast<double>(x)));
      else
        return std::atan2(y, x);
    }
#endif
    LSTREF_UNARY(sin)
    LSTREF_UNARY(cos)
    LSTREF_UNARY(tan)
    LSTREF_UNARY(asin)
    LSTREF_UNARY(acos)
    LSTREF_UNARY(atan)
    LSTREF_UNARY(sinh)
    LSTREF_UNARY(acosh)
    LSTREF_UNARY(exp)
    LSTREF_UNARY(log)
#undef LSTREF_UNARY
  }  // namespace math

}  // namespace alpaka
