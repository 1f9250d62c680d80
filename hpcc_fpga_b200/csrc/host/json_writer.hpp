// Minimal ordered JSON value and writer for the result dump
// (the reference uses nlohmann::json, shared/include/hpcc_benchmark.hpp:490-516).
#pragma once

#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace hpcc_base {

class Json {
public:
    enum class Kind { Null, Bool, Number, String, Array, Object };

    Json() = default;
    static Json boolean(bool v) { Json j; j.kind_ = Kind::Bool; j.b_ = v; return j; }
    static Json number(double v) { Json j; j.kind_ = Kind::Number; j.d_ = v; return j; }
    static Json integer(long long v) { Json j; j.kind_ = Kind::Number; j.d_ = (double)v; j.int_ = true; return j; }
    static Json string(const std::string& v) { Json j; j.kind_ = Kind::String; j.s_ = v; return j; }
    static Json array() { Json j; j.kind_ = Kind::Array; return j; }
    static Json object() { Json j; j.kind_ = Kind::Object; return j; }

    Json& operator[](const std::string& key) {
        if (kind_ != Kind::Object) { kind_ = Kind::Object; }
        return obj_[key];
    }
    void push_back(const Json& v) {
        if (kind_ != Kind::Array) kind_ = Kind::Array;
        arr_.push_back(v);
    }
    bool contains(const std::string& key) const { return kind_ == Kind::Object && obj_.count(key) > 0; }

    std::string dump() const {
        std::ostringstream os;
        write(os);
        return os.str();
    }

private:
    static void escape(std::ostream& os, const std::string& s) {
        os << '"';
        for (char c : s) {
            switch (c) {
                case '"': os << "\\\""; break;
                case '\\': os << "\\\\"; break;
                case '\n': os << "\\n"; break;
                case '\t': os << "\\t"; break;
                case '\r': os << "\\r"; break;
                default:
                    if ((unsigned char)c < 0x20) {
                        char buf[8];
                        std::snprintf(buf, sizeof(buf), "\\u%04x", (unsigned char)c);
                        os << buf;
                    } else {
                        os << c;
                    }
            }
        }
        os << '"';
    }
    void write(std::ostream& os) const {
        switch (kind_) {
            case Kind::Null: os << "null"; break;
            case Kind::Bool: os << (b_ ? "true" : "false"); break;
            case Kind::Number:
                if (!std::isfinite(d_)) {
                    os << "null";
                } else if (int_) {
                    os << (long long)d_;
                } else {
                    char buf[40];
                    std::snprintf(buf, sizeof(buf), "%.17g", d_);
                    os << buf;
                }
                break;
            case Kind::String: escape(os, s_); break;
            case Kind::Array: {
                os << '[';
                for (size_t i = 0; i < arr_.size(); i++) {
                    if (i) os << ',';
                    arr_[i].write(os);
                }
                os << ']';
                break;
            }
            case Kind::Object: {
                os << '{';
                bool first = true;
                for (const auto& kv : obj_) {
                    if (!first) os << ',';
                    first = false;
                    escape(os, kv.first);
                    os << ':';
                    kv.second.write(os);
                }
                os << '}';
                break;
            }
        }
    }

    Kind kind_ = Kind::Null;
    bool b_ = false;
    bool int_ = false;
    double d_ = 0.0;
    std::string s_;
    std::vector<Json> arr_;
    std::map<std::string, Json> obj_;
};

}  // namespace hpcc_base
