#pragma once
// Command-line handling for the GraphOne apps.  The apps use a small part of
// CLI11's interface (CLI::App::add_option / add_flag / ->required(),
// CLI11_PARSE); this is an independent implementation of just that part,
// plus GraphOne's add_common_args (reference: utils/cli.hpp:18-32).

#include <functional>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "GraphOne/loader/opts.hpp"

namespace CLI {

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
    const std::vector<std::string>& names() const { return names_; }
    const std::string& desc() const { return desc_; }
    bool flag() const { return flag_; }
    bool is_required() const { return required_; }
    bool seen = false;
    bool assign(const std::string& v) { return set_(v); }

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
        opts_.emplace_back(new Option(split(names), desc, false, [&target](const std::string& v) {
            std::istringstream is(v);
            T tmp{};
            if constexpr (std::is_same_v<T, std::string>) {
                target = v;
                return true;
            } else {
                is >> tmp;
                if (is.fail()) return false;
                target = tmp;
                return true;
            }
        }));
        return opts_.back().get();
    }

    Option* add_flag(const std::string& names, bool& target, const std::string& desc = "") {
        opts_.emplace_back(new Option(split(names), desc, true, [&target](const std::string&) {
            target = true;
            return true;
        }));
        return opts_.back().get();
    }

    // Returns -1 when the program should continue, else its exit code.
    int parse(int argc, char** argv) {
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a == "-h" || a == "--help") {
                help(std::cout, argv[0]);
                return 0;
            }
            std::string value;
            bool inline_value = false;
            const auto eq = a.find('=');
            if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
                value = a.substr(eq + 1);
                a = a.substr(0, eq);
                inline_value = true;
            }
            Option* o = find(a);
            if (!o) {
                std::cerr << "unknown argument: " << a << "\n";
                return 109;
            }
            o->seen = true;
            if (o->flag()) {
                o->assign("1");
                continue;
            }
            if (!inline_value) {
                if (i + 1 >= argc) {
                    std::cerr << a << ": missing value\n";
                    return 109;
                }
                value = argv[++i];
            }
            if (!o->assign(value)) {
                std::cerr << a << ": cannot parse '" << value << "'\n";
                return 109;
            }
        }
        for (auto& o : opts_) {
            if (o->is_required() && !o->seen) {
                std::cerr << o->names().back() << " is required\n";
                return 106;
            }
        }
        return -1;
    }

private:
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
#define CLI11_PARSE(app, argc, argv)                 \
    do {                                             \
        const int g1_cli_rc_ = (app).parse((argc), (argv)); \
        if (g1_cli_rc_ >= 0) return g1_cli_rc_;      \
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
