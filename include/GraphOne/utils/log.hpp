#pragma once
// Console output of the GraphOne API (reference: utils/log.hpp:31-63):
// printx prints its arguments then a newline, LOG_ERROR prints and exits(1),
// LOG_DEBUG prints only when DEBUG_LOG is defined.  Objects with a
// ToString() member print through it.

#include <cstdlib>
#include <iostream>
#include <string>
#include <type_traits>

#include "GraphOne/utils/string.hpp"

namespace graph_one {

namespace detail {
template <typename T>
decltype(auto) printable(const T& v) {
    if constexpr (std::is_class_v<T> && utils::HasToStrMethod<T>::value)
        return v.ToString();
    else
        return (v);
}

template <typename... Ts>
void emit_line(std::ostream& os, const char* label, Ts&&... args) {
    os << label;
    (os << ... << printable(args));
    os << std::endl;
}
}  // namespace detail

template <typename... Ts>
void printx(Ts&&... args) {
    detail::emit_line(std::cout, "", std::forward<Ts>(args)...);
}

template <typename... Ts>
void LOG_INFO(Ts&&... args) {
    detail::emit_line(std::cout, "[INFO]  ", std::forward<Ts>(args)...);
}

template <typename... Ts>
void LOG_WARNING(Ts&&... args) {
    detail::emit_line(std::cout, "[WARN]  ", std::forward<Ts>(args)...);
}

template <typename... Ts>
[[noreturn]] void LOG_ERROR(Ts&&... args) {
    detail::emit_line(std::cout, "[ERROR] ", std::forward<Ts>(args)...);
    std::exit(1);
}

template <typename... Ts>
void LOG_DEBUG(Ts&&... args) {
#ifdef DEBUG_LOG
    detail::emit_line(std::cout, "[DEBUG] ", std::forward<Ts>(args)...);
#else
    ((void)args, ...);
#endif
}

}  // namespace graph_one
