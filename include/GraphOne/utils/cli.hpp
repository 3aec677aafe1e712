#pragma once
// Command-line handling for the GraphOne apps.  The apps use a small part of
// CLI11's interface (CLI::App::add_option / add_flag / ->required(),
// CLI11_PARSE); this is an independent implementation of just that part,
// plus GraphOne's add_common_args (reference: utils/cli.hpp:18-32).
//
// Accepted forms, as CLI11 2.3 (the version GraphOne vendors) reads them:
//   --name value, --name=value (an empty "=value" takes the next argument),
//   -n value, -nvalue, and combined short flags (-dr, -dri value);
//   the argument after an option is its value even when it starts with '-';
//   "--" ends the options (what follows is positional).
// Values: unsigned integers in decimal, 0x hex, 0b binary or leading-0
// octal, no sign but '+', the whole argument; floating point via strtold,
// the whole argument; an empty number is zero; a flag given "=value" takes true/t/yes/y/on/enable/+/
// or a positive number for true, false/f/no/n/off/disable/- or a number <= 0
// for false (case-insensitive), an empty value meaning true.
// Exit codes (CLI11's): 0 after --help, 104 a value that does not convert,
// 106 a required option missing, 109 an unexpected argument, 114 a missing
// value or a single-value option given twice.  Conversion and count errors
// come first (in declaration order), then required options, then unexpected
// arguments.

#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdlib>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "GraphOne/loader/opts.hpp"

namespace CLI {

namespace detail {

// Parses the whole of s as an unsigned integer (see above).
inline bool parse_unsigned(const std::string& s, unsigned long long* out) {
    size_t i = 0;
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    if (i < s.size() && s[i] == '-') return false;
    if (i < s.size() && s[i] == '+') ++i;
    if (i >= s.size()) return false;
    int base = 0;
    if (s.size() - i > 2 && s[i] == '0' && (s[i + 1] == 'b' || s[i + 1] == 'B')) {
        base = 2;
        i += 2;
    }
    if (i >= s.size() || !std::isalnum((unsigned char)s[i])) return false;
    const char* b = s.c_str() + i;
    char* end = nullptr;
    errno = 0;
    const unsigned long long v = std::strtoull(b, &end, base);
    if (errno == ERANGE || end == b || end != s.c_str() + s.size()) return false;
    *out = v;
    return true;
}

inline bool parse_signed(const std::string& s, long long* out) {
    size_t i = 0;
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    bool neg = false;
    if (i < s.size() && (s[i] == '-' || s[i] == '+')) neg = s[i++] == '-';
    unsigned long long mag = 0;
    if (i >= s.size() || s[i] == '+' || s[i] == '-' || !parse_unsigned(s.substr(i), &mag)) return false;
    const unsigned long long lim = (unsigned long long)std::numeric_limits<long long>::max() + (neg ? 1 : 0);
    if (mag > lim) return false;
    *out = neg ? (long long)(0ull - mag) : (long long)mag;
    return true;
}

inline bool parse_floating(const std::string& s, long double* out) {
    if (s.empty()) return false;
    char* end = nullptr;
    const long double v = std::strtold(s.c_str(), &end);
    if (end == s.c_str() || end != s.c_str() + s.size()) return false;
    *out = v;
    return true;
}

// The value of "--flag=s": 1 true, 0 false, -1 not a flag value.
inline int parse_flag_value(const std::string& s) {
    if (s.empty()) return 1;
    std::string l;
    for (char c : s) l += (char)std::tolower((unsigned char)c);
    for (const char* w : {"true", "t", "yes", "y", "on", "enable", "+"})
        if (l == w) return 1;
    for (const char* w : {"false", "f", "no", "n", "off", "disable", "-"})
        if (l == w) return 0;
    // otherwise the leading decimal integer decides (the rest is ignored)
    char* end = nullptr;
    errno = 0;
    const long long v = std::strtoll(s.c_str(), &end, 10);
    if (end == s.c_str() || errno == ERANGE) return -1;
    return v > 0 ? 1 : 0;
}

template <typename T>
bool convert(const std::string& s, T& target) {
    if constexpr (std::is_same_v<T, std::string>) {
        target = s;
        return true;
    } else if constexpr (std::is_same_v<T, bool>) {
        const int f = parse_flag_value(s);
        if (f < 0) return false;
        target = f == 1;
        return true;
    } else if (s.empty()) {  // an empty number is zero
        target = T{};
        return true;
    } else if constexpr (std::is_integral_v<T> && std::is_unsigned_v<T>) {
        unsigned long long v = 0;
        if (!parse_unsigned(s, &v) || v > (unsigned long long)std::numeric_limits<T>::max()) return false;
        target = (T)v;
        return true;
    } else if constexpr (std::is_integral_v<T>) {
        long long v = 0;
        if (!parse_signed(s, &v) || v < (long long)std::numeric_limits<T>::min() ||
            v > (long long)std::numeric_limits<T>::max())
            return false;
        target = (T)v;
        return true;
    } else if constexpr (std::is_floating_point_v<T>) {
        long double v = 0;
        if (!parse_floating(s, &v)) return false;
        const long double hi = std::numeric_limits<T>::max();
        if (v > hi || v < -hi)  // beyond the type's range: infinity, like IEEE rounding
            target = v > 0 ? std::numeric_limits<T>::infinity() : -std::numeric_limits<T>::infinity();
        else
            target = (T)v;
        return true;
    } else {
        static_assert(std::is_same_v<T, std::string>, "unsupported option type");
        return false;
    }
}

}  // namespace detail

class Option {
public:
    Option(std::vector<std::string> names, std::string desc, bool flag,
           std::function<bool(const std::string&)> set)
        : names_(std::move(names)), desc_(std::move(desc)), flag_(flag), set_(std::move(set)) {}
    Option* required(bool r = true) {
        required_ = r;
        return this;
    }
    bool matches(const std::string& arg) const {
        for (auto& n : names_)
            if (n == arg) return true;
        return false;
    }
    // The long name when there is one (used in messages).
    const std::string& name() const {
        for (auto& n : names_)
            if (n.rfind("--", 0) == 0) return n;
        return names_.back();
    }
    const std::vector<std::string>& names() const { return names_; }
    const std::string& desc() const { return desc_; }
    bool flag() const { return flag_; }
    bool is_required() const { return required_; }
    bool assign(const std::string& v) { return set_(v); }

    // Values met on the command line (flags: "" for a bare flag).
    std::vector<std::string> given;
    bool missing_value = false;

private:
    std::vector<std::string> names_;
    std::string desc_;
    bool flag_;
    bool required_ = false;
    std::function<bool(const std::string&)> set_;
};

class App {
public:
    explicit App(std::string description = "") : desc_(std::move(description)) {}

    template <typename T>
    Option* add_option(const std::string& names, T& target, const std::string& desc = "") {
        opts_.emplace_back(new Option(split(names), desc, false,
                                      [&target](const std::string& v) { return detail::convert(v, target); }));
        return opts_.back().get();
    }

    Option* add_flag(const std::string& names, bool& target, const std::string& desc = "") {
        opts_.emplace_back(new Option(split(names), desc, true, [&target](const std::string& v) {
            const int f = detail::parse_flag_value(v);
            if (f < 0) return false;
            target = f == 1;
            return true;
        }));
        return opts_.back().get();
    }

    // Returns -1 when the program should continue, else its exit code.
    int parse(int argc, char** argv) {
        std::vector<std::string> extras;
        bool help_asked = false;
        bool positional_only = false;
        for (int i = 1; i < argc; ++i) {
            const std::string a = argv[i];
            if (positional_only || a.size() < 2 || a[0] != '-' || a == "-") {
                extras.push_back(a);
                continue;
            }
            if (a == "--") {
                positional_only = true;
                continue;
            }
            if (a == "-h" || a == "--help") {
                help_asked = true;
                continue;
            }
            if (a[1] == '-') {  // --name or --name=value
                const auto eq = a.find('=');
                Option* o = find(a.substr(0, eq));
                if (!o) {
                    extras.push_back(a);
                    continue;
                }
                if (eq != std::string::npos && (o->flag() || eq + 1 < a.size())) {
                    o->given.push_back(a.substr(eq + 1));
                } else if (o->flag()) {
                    o->given.emplace_back();
                } else {
                    take_next(o, argc, argv, &i);
                }
                continue;
            }
            // -x, -xvalue, -xyz (combined short flags)
            for (size_t k = 1; k < a.size(); ++k) {
                Option* o = find(std::string("-") + a[k]);
                if (!o && a[k] == 'h') {
                    help_asked = true;
                    continue;
                }
                if (!o) {
                    extras.push_back(std::string("-") + a.substr(k));
                    break;
                }
                if (o->flag()) {
                    o->given.emplace_back();
                    continue;
                }
                if (k + 1 < a.size())
                    o->given.push_back(a.substr(k + 1));
                else
                    take_next(o, argc, argv, &i);
                break;
            }
        }
        for (auto& o : opts_) {
            if (o->missing_value) {
                std::cerr << o->name() << ": 1 required value missing\n";
                return 114;
            }
            if (!o->flag() && o->given.size() > 1) {
                std::cerr << o->name() << ": at most 1 value expected, received " << o->given.size() << "\n";
                return 114;
            }
            for (auto& v : o->given)
                if (!o->assign(v)) {
                    std::cerr << "Could not convert: " << o->name() << " = " << v << "\n";
                    return 104;
                }
        }
        if (help_asked) {
            help(std::cout, argv[0]);
            return 0;
        }
        for (auto& o : opts_)
            if (o->is_required() && o->given.empty()) {
                std::cerr << o->name() << " is required\n";
                return 106;
            }
        if (!extras.empty()) {
            std::cerr << "The following argument was not expected:";
            for (auto& e : extras) std::cerr << " " << e;
            std::cerr << "\n";
            return 109;
        }
        return -1;
    }

private:
    static void take_next(Option* o, int argc, char** argv, int* i) {
        if (*i + 1 < argc)
            o->given.push_back(argv[++*i]);
        else
            o->missing_value = true;
    }
    static std::vector<std::string> split(const std::string& names) {
        std::vector<std::string> out;
        std::string cur;
        for (char c : names) {
            if (c == ',') {
                if (!cur.empty()) out.push_back(cur);
                cur.clear();
            } else {
                cur += c;
            }
        }
        if (!cur.empty()) out.push_back(cur);
        return out;
    }
    Option* find(const std::string& a) {
        for (auto& o : opts_)
            if (o->matches(a)) return o.get();
        return nullptr;
    }
    void help(std::ostream& os, const char* prog) const {
        os << (desc_.empty() ? prog : desc_) << "\nOptions:\n";
        for (auto& o : opts_) {
            os << "  ";
            for (size_t k = 0; k < o->names().size(); ++k) os << (k ? "," : "") << o->names()[k];
            os << "  " << o->desc() << (o->is_required() ? " (required)" : "") << "\n";
        }
    }
    std::string desc_;
    std::vector<std::unique_ptr<Option>> opts_;
};

}  // namespace CLI

// Parses the command line; returns from main with the exit code on --help or
// on an error.
#define CLI11_PARSE(app, argc, argv)                        \
    do {                                                    \
        const int g1_cli_rc_ = (app).parse((argc), (argv)); \
        if (g1_cli_rc_ >= 0) return g1_cli_rc_;             \
    } while (0)

namespace graph_one {

inline void add_common_args(CLI::App& app, std::string& input_graph, std::string& output_path,
                            bool& reorder_vid, LoadEdgeOpts& opts) {
    app.add_option("-i,--input_graph", input_graph, "input graph dataset file")->required();
    app.add_option("-o,--output", output_path, "output path to save result");
    app.add_flag("-r,--reorder", reorder_vid, "reorder vertex id in graph dataset to compress");
    app.add_option("--file_ext", opts.file_ext, "graph dataset file extension");
    app.add_option("--comment_prefix", opts.comment_prefix, "graph dataset file comment line prefix");
    app.add_option("--line_sep", opts.line_sep, "graph dataset file line data delimiter");
    app.add_flag("-d,--is_directed", opts.is_directed, "directed graph dataset");
    app.add_flag("--keep_self", opts.keep_self_loop, "keep self loop edges in graph");
    app.add_flag("--keep_dup", opts.keep_duplicate_edges, "keep duplicate edges in graph");
}

}  // namespace graph_one
