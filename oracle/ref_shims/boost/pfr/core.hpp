#pragma once
// Minimal stand-in for boost::pfr::tuple_size_v / tuple_element_t over aggregates (C++20).
#include <cstddef>
#include <tuple>
#include <type_traits>
#include <utility>
namespace boost { namespace pfr { namespace detail {
struct any_init { template<class U> operator U() const; };
template<class T, std::size_t... I>
constexpr bool braces_ok(std::index_sequence<I...>) { return requires { T{((void)I, any_init{})...}; }; }
template<class T, std::size_t N = 0>
constexpr std::size_t count_fields() {
  if constexpr (N > 64) return 0;
  else if constexpr (braces_ok<T>(std::make_index_sequence<N + 1>{})) return count_fields<T, N + 1>();
  else return N;
}
}}}
#include "core_cases.hpp"
namespace boost { namespace pfr {
template<class T> inline constexpr std::size_t tuple_size_v = detail::count_fields<T>();
template<class T> struct tuple_size : std::integral_constant<std::size_t, tuple_size_v<T>> {};
template<std::size_t I, class T>
using tuple_element_t = std::tuple_element_t<I, typename decltype(detail::member_types<T, tuple_size_v<T>>(std::declval<T&>()))::type>;
}}
