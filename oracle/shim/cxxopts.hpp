// Minimal stand-in for the cxxopts option parser (jarro2783/cxxopts v2.2.1 API
// surface), written for this project so that the reference's CPU executables
// can be compiled from their unmodified sources into oracle/_ref/ without the
// network fetch their CMakeLists.txt performs.  Only what those sources use:
// Options(name, help), add_options()(name, desc[, value]), value<T>(T&),
// parse(argc, argv) -> result.count(name), help(), OptionException.
//
// Test infrastructure only (oracle build); never part of the product.
#ifndef SI_ORACLE_CXXOPTS_SHIM_HPP
#define SI_ORACLE_CXXOPTS_SHIM_HPP

#include <exception>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace cxxopts {

class OptionException : public std::exception {
public:
    explicit OptionException(std::string m) : msg_(std::move(m)) {}
    const char* what() const noexcept override { return msg_.c_str(); }
private:
    std::string msg_;
};

struct ValueBase {
    virtual ~ValueBase() = default;
    virtual void parse(const std::string& text) = 0;
    virtual bool is_flag() const { return false; }
};

template <class T>
struct TypedValue : ValueBase {
    T own{};
    T* target;
    explicit TypedValue(T* t) : target(t ? t : &own) {}
    void parse(const std::string& text) override {
        std::istringstream in(text);
        T v{};
        in >> v;
        if (in.fail() || !in.eof()) throw OptionException("Argument '" + text + "' failed to parse");
        *target = v;
    }
};

template <>
struct TypedValue<std::string> : ValueBase {
    std::string own;
    std::string* target;
    explicit TypedValue(std::string* t) : target(t ? t : &own) {}
    void parse(const std::string& text) override { *target = text; }
};

template <>
struct TypedValue<bool> : ValueBase {
    bool own = false;
    bool* target;
    explicit TypedValue(bool* t) : target(t ? t : &own) {}
    bool is_flag() const override { return true; }
    void parse(const std::string& text) override {
        if (text.empty() || text == "true" || text == "1" || text == "yes") *target = true;
        else if (text == "false" || text == "0" || text == "no") *target = false;
        else throw OptionException("Argument '" + text + "' failed to parse");
    }
};

template <class T>
std::shared_ptr<ValueBase> value(T& t) { return std::make_shared<TypedValue<T>>(&t); }
template <class T>
std::shared_ptr<ValueBase> value() { return std::make_shared<TypedValue<T>>(nullptr); }

class ParseResult {
public:
    size_t count(const std::string& name) const {
        auto it = counts_.find(name);
        return it == counts_.end() ? 0 : it->second;
    }
    std::map<std::string, size_t> counts_;
};

class Options;

class OptionAdder {
public:
    explicit OptionAdder(Options& o) : o_(o) {}
    OptionAdder& operator()(const std::string& name, const std::string& desc,
                            std::shared_ptr<ValueBase> v = nullptr);
private:
    Options& o_;
};

class Options {
public:
    Options(std::string program, std::string help) : program_(std::move(program)), help_(std::move(help)) {}
    OptionAdder add_options() { return OptionAdder(*this); }

    ParseResult parse(int& argc, char**& argv) {
        ParseResult r;
        for (int i = 1; i < argc; ++i) {
            std::string arg = argv[i];
            if (arg.size() < 3 || arg[0] != '-' || arg[1] != '-') continue;  // positional: ignored
            std::string name = arg.substr(2), text;
            bool has_text = false;
            auto eq = name.find('=');
            if (eq != std::string::npos) { text = name.substr(eq + 1); name = name.substr(0, eq); has_text = true; }
            auto it = opts_.find(name);
            if (it == opts_.end()) throw OptionException("Option '" + name + "' does not exist");
            auto& v = it->second.value;
            if (v) {
                if (!has_text && !v->is_flag()) {
                    if (i + 1 >= argc) throw OptionException("Option '" + name + "' is missing an argument");
                    text = argv[++i];
                }
                v->parse(text);
            }
            r.counts_[name] += 1;
        }
        return r;
    }

    std::string help() const {
        std::ostringstream out;
        out << help_ << "\nUsage:\n  " << program_ << " [OPTION...]\n\n";
        for (const auto& name : order_) out << "      --" << name << "  " << opts_.at(name).desc << "\n";
        return out.str();
    }

private:
    friend class OptionAdder;
    struct Entry { std::string desc; std::shared_ptr<ValueBase> value; };
    std::string program_, help_;
    std::map<std::string, Entry> opts_;
    std::vector<std::string> order_;
};

inline OptionAdder& OptionAdder::operator()(const std::string& name, const std::string& desc,
                                            std::shared_ptr<ValueBase> v) {
    o_.opts_[name] = Options::Entry{desc, std::move(v)};
    o_.order_.push_back(name);
    return *this;
}

}  // namespace cxxopts

#endif
