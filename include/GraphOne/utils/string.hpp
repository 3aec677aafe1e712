#pragma once
// String helpers of the GraphOne API (reference: utils/string.hpp).  The apps
// and the loader call StrEndWith / StrStartWith / StrStrip and the ToString
// family; containers print themselves through their own ToString() member.

#include <string>
#include <vector>
#include <sstream>
#include <utility>
#include <unordered_map>
#include <type_traits>

#include "GraphOne/type.hpp"

namespace graph_one::utils {

inline bool StrEndWith(const std::string& str, const std::string& suffix) {
    return str.size() >= suffix.size() &&
           str.compare(str.size() - suffix.size(), suffix.size(), suffix) == 0;
}

inline bool StrStartWith(const std::string& str, const std::string& prefix) {
    return str.size() >= prefix.size() && str.compare(0, prefix.size(), prefix) == 0;
}

inline std::string StrStrip(const std::string& str, const std::string& chars = " \t\n\r") {
    const auto first = str.find_first_not_of(chars);
    if (first == std::string::npos) return std::string();
    const auto last = str.find_last_not_of(chars);
    return str.substr(first, last - first + 1);
}

template <typename T, typename = void>
struct HasToStrMethod : std::false_type {};

template <typename T>
struct HasToStrMethod<T, std::void_t<decltype(std::declval<const T&>().ToString())>>
    : std::true_type {};

template <typename T>
std::string NumToString(T num) {
    std::ostringstream os;
    os << +num;
    return os.str();
}

template <typename T>
std::string ToString(const T& x) {
    if constexpr (std::is_same_v<T, bool>) {
        return x ? "true" : "false";
    } else if constexpr (std::is_same_v<T, arch_t>) {
        return x == arch_t::cpu ? "cpu" : "cuda";
    } else if constexpr (std::is_arithmetic_v<T>) {
        return NumToString(x);
    } else if constexpr (HasToStrMethod<T>::value) {
        return x.ToString();
    } else if constexpr (std::is_convertible_v<T, std::string>) {
        return std::string(x);
    } else {
        std::ostringstream os;
        os << x;
        return os.str();
    }
}

template <typename K, typename V>
std::string ToString(const std::pair<K, V>& p) {
    return "(" + ToString(p.first) + "," + ToString(p.second) + ")";
}

// "[a,b,c]"; str_func formats one element (default ToString).
template <typename T, typename F>
std::string VecToString(const T* vec, size_t size, F str_func) {
    std::string str = "[";
    for (size_t i = 0; i < size; ++i) {
        if (i) str += ",";
        str += str_func(vec[i]);
    }
    return str + "]";
}

template <typename T>
std::string VecToString(const T* vec, size_t size) {
    return VecToString(vec, size, [](const T& x) { return ToString(x); });
}

template <typename T, typename F>
std::string VecToString(const std::vector<T>& vec, F str_func) {
    return VecToString(vec.data(), vec.size(), str_func);
}

template <typename T>
std::string VecToString(const std::vector<T>& vec) {
    return VecToString(vec.data(), vec.size());
}

template <typename K, typename V, typename F>
std::string HashmapToString(const std::unordered_map<K, V>& hashmap, F str_func) {
    std::string str = "[";
    bool first = true;
    for (const auto& kv : hashmap) {
        if (!first) str += ",";
        first = false;
        str += str_func(kv);
    }
    return str + "]";
}

template <typename K, typename V>
std::string HashmapToString(const std::unordered_map<K, V>& hashmap) {
    return HashmapToString(hashmap, [](const std::pair<const K, V>& kv) { return ToString(kv); });
}

}  // namespace graph_one::utils
