#pragma once
#include <string>
#include <stdexcept>
#include <ostream>
namespace nlohmann {
namespace detail { struct type_error : std::runtime_error { using std::runtime_error::runtime_error; }; }
struct json { json() {} template<class T> json(const T&) {} template<class T> T get() const { return T{}; }
  template<class T> operator T() const { return T{}; }
  std::string dump(int = -1) const { return {}; } using type_error = detail::type_error; };
inline std::ostream& operator<<(std::ostream& o, const json&) { return o; }
}
