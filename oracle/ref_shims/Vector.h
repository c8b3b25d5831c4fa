#pragma once
#include <array>
#include <cstddef>
#include <cmath>
#include <cstdint>
namespace ref_shim {
template<typename T, unsigned N> struct Mask {
  std::array<bool, N> v{};
  Mask() = default;
  explicit Mask(const bool* p) { for (unsigned i = 0; i < N; ++i) v[i] = p[i]; }
  bool hlor() const { for (unsigned i = 0; i < N; ++i) if (v[i]) return true; return false; }
  Mask operator&&(const Mask& o) const { Mask r; for (unsigned i = 0; i < N; ++i) r.v[i] = v[i] && o.v[i]; return r; }
  bool operator[](unsigned i) const { return v[i]; }
  static constexpr std::size_t length() { return N; }
};
template<typename T, unsigned N> struct Vec {
  std::array<T, N> v{};
  Vec() = default;
  Vec(T s) { v.fill(s); }
  explicit Vec(const T* p) { for (unsigned i = 0; i < N; ++i) v[i] = p[i]; }
  static constexpr std::size_t length() { return N; }
  T operator[](unsigned i) const { return v[i]; }
#define SHIM_BINOP(OP) \
  friend Vec operator OP(const Vec& a, const Vec& b) { Vec r; for (unsigned i = 0; i < N; ++i) r.v[i] = a.v[i] OP b.v[i]; return r; } \
  friend Vec operator OP(const Vec& a, T b) { Vec r; for (unsigned i = 0; i < N; ++i) r.v[i] = a.v[i] OP b; return r; } \
  friend Vec operator OP(T a, const Vec& b) { Vec r; for (unsigned i = 0; i < N; ++i) r.v[i] = a OP b.v[i]; return r; }
  SHIM_BINOP(+) SHIM_BINOP(-) SHIM_BINOP(*) SHIM_BINOP(/)
#undef SHIM_BINOP
  friend Mask<T, N> operator<(const Vec& a, T b) { Mask<T, N> r; for (unsigned i = 0; i < N; ++i) r.v[i] = a.v[i] < b; return r; }
  Mask<T, N> cmple(T b) const { Mask<T, N> r; for (unsigned i = 0; i < N; ++i) r.v[i] = v[i] <= b; return r; }
  Vec blend(const Mask<T, N>& m, const Vec& b) const { Vec r; for (unsigned i = 0; i < N; ++i) r.v[i] = m.v[i] ? b.v[i] : v[i]; return r; }
  Vec abs() const { Vec r; for (unsigned i = 0; i < N; ++i) r.v[i] = std::fabs(v[i]); return r; }
  Vec copysign(const Vec& b) const { Vec r; for (unsigned i = 0; i < N; ++i) r.v[i] = std::copysign(v[i], b.v[i]); return r; }
  unsigned imin(const Mask<T, N>& m) const { unsigned best = 0; bool have = false; for (unsigned i = 0; i < N; ++i) if (m.v[i] && (!have || v[i] < v[best])) { best = i; have = true; } return best; }
};
} // namespace ref_shim
namespace Allen { namespace device {
template<typename T> struct Vector128_sel { using t = ref_shim::Vec<T, 16 / sizeof(float)>; };
template<> struct Vector128_sel<bool> { using t = ref_shim::Mask<float, 4>; };
template<typename T> using Vector128 = typename Vector128_sel<T>::t;
template<typename T> using Vector = Vector128<T>;
template<typename T = float> constexpr std::size_t vector128_length() { return 4; }
template<typename T = float> constexpr std::size_t vector_length() { return 4; }
}}
template<typename T, unsigned N>
inline ref_shim::Vec<T, N> signselect(const ref_shim::Vec<T, N>& x, const ref_shim::Vec<T, N>& a, const ref_shim::Vec<T, N>& b) { return a.blend(x.cmple(0.f), b); }
template<unsigned N> inline ref_shim::Vec<float, N> fabsf(const ref_shim::Vec<float, N>& v) { return v.abs(); }
template<typename T, unsigned N> inline ref_shim::Vec<T, N> copysignf(const ref_shim::Vec<T, N>& a, const ref_shim::Vec<T, N>& b) { return a.copysign(b); }
