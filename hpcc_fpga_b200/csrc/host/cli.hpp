// Command-line options in the style the reference declares them with cxxopts
// (shared/include/hpcc_benchmark.hpp:254-297, linpack_benchmark.hpp:60-71):
// "f,file" style names (short,long), options with or without a value,
// defaults, "-x value", "-xvalue", "--name value" and "--name=value".
#pragma once

#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace hpcc_base {

class OptionError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

class Options {
public:
    struct Spec {
        std::string shortname, longname, help, def;
        bool has_value = false, has_default = false;
    };

    explicit Options(std::string program, std::string description = "")
        : program_(std::move(program)), description_(std::move(description)) {}

    // names: "f,file" or "n" or "skip-validation"
    Options& add(const std::string& names, const std::string& help, bool has_value = false,
                 const std::string& def = "", bool has_default = false) {
        Spec s;
        const auto comma = names.find(',');
        if (comma != std::string::npos) {
            s.shortname = names.substr(0, comma);
            s.longname = names.substr(comma + 1);
        } else if (names.size() == 1) {
            s.shortname = names;
        } else {
            s.longname = names;
        }
        s.help = help;
        s.has_value = has_value;
        s.def = def;
        s.has_default = has_default;
        specs_.push_back(s);
        return *this;
    }
    Options& value(const std::string& names, const std::string& help, const std::string& def) {
        return add(names, help, true, def, true);
    }
    Options& value(const std::string& names, const std::string& help) { return add(names, help, true); }
    Options& flag(const std::string& names, const std::string& help) { return add(names, help, false); }

    class Result {
    public:
        size_t count(const std::string& k) const { return given_.count(k) ? given_.at(k) : 0; }
        bool has(const std::string& k) const { return values_.count(k) > 0; }
        std::string str(const std::string& k) const {
            auto it = values_.find(k);
            if (it == values_.end()) throw OptionError("Option '" + k + "' has no value");
            return it->second;
        }
        long long integer(const std::string& k) const {
            const std::string v = str(k);
            size_t pos = 0;
            long long x = 0;
            try {
                x = std::stoll(v, &pos);
            } catch (...) {
                throw OptionError("Argument '" + v + "' failed to parse for option '" + k + "'");
            }
            if (pos != v.size()) throw OptionError("Argument '" + v + "' failed to parse for option '" + k + "'");
            return x;
        }
        double real(const std::string& k) const {
            const std::string v = str(k);
            try {
                return std::stod(v);
            } catch (...) {
                throw OptionError("Argument '" + v + "' failed to parse for option '" + k + "'");
            }
        }
        std::map<std::string, std::string> values_;
        std::map<std::string, size_t> given_;
    };

    Result parse(int argc, char const* const* argv) const {
        Result r;
        for (const auto& s : specs_)
            if (s.has_default) store(r, s, s.def, false);
        for (int i = 1; i < argc; i++) {
            std::string a = argv[i];
            const Spec* s = nullptr;
            std::string val;
            bool inline_val = false;
            if (a.rfind("--", 0) == 0) {
                std::string name = a.substr(2);
                const auto eq = name.find('=');
                if (eq != std::string::npos) {
                    val = name.substr(eq + 1);
                    name = name.substr(0, eq);
                    inline_val = true;
                }
                s = find(name);
                if (s == nullptr) throw OptionError("Option '" + name + "' does not exist");
            } else if (a.size() >= 2 && a[0] == '-') {
                s = find(a.substr(1, 1));
                if (s == nullptr) throw OptionError("Option '" + a.substr(1, 1) + "' does not exist");
                if (a.size() > 2) {
                    val = a.substr(2);
                    inline_val = true;
                }
            } else {
                continue;  // positional arguments are ignored, as with cxxopts' default
            }
            if (s->has_value) {
                if (!inline_val) {
                    if (i + 1 >= argc) throw OptionError("Option '" + key(*s) + "' is missing an argument");
                    val = argv[++i];
                }
                store(r, *s, val, true);
            } else {
                if (inline_val) throw OptionError("Option '" + key(*s) + "' does not take an argument");
                store(r, *s, "", true);
            }
        }
        return r;
    }

    std::string help() const {
        std::ostringstream os;
        os << description_ << "Usage:\n  " << program_ << " [OPTION...]\n\n";
        for (const auto& s : specs_) {
            std::string n = "  ";
            n += s.shortname.empty() ? "    " : "-" + s.shortname + (s.longname.empty() ? "" : ", ");
            if (!s.longname.empty()) n += "--" + s.longname;
            if (s.has_value) n += " arg";
            os << n;
            for (size_t k = n.size(); k < 30; k++) os << ' ';
            os << ' ' << s.help;
            if (s.has_default) os << " (default: " << s.def << ")";
            os << "\n";
        }
        return os.str();
    }

private:
    static std::string key(const Spec& s) { return s.longname.empty() ? s.shortname : s.longname; }
    const Spec* find(const std::string& name) const {
        for (const auto& s : specs_)
            if (s.shortname == name || s.longname == name) return &s;
        return nullptr;
    }
    static void store(Result& r, const Spec& s, const std::string& v, bool given) {
        for (const std::string& k : {s.shortname, s.longname}) {
            if (k.empty()) continue;
            r.values_[k] = v;
            if (given) r.given_[k]++;
        }
    }

    std::string program_, description_;
    std::vector<Spec> specs_;
};

}  // namespace hpcc_base
