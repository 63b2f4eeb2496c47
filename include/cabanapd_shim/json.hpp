// Minimal JSON reader for CabanaPD input decks ({"key": {"value": ...,
// "unit": ...}}): objects, arrays, numbers, strings, booleans, null.
#pragma once

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace cabanapd_shim {

class Json {
  public:
    enum Kind { Null, Bool, Number, String, Array, Object };

    Json() = default;
    explicit Json(double v) : kind_(Number), num_(v) {}
    explicit Json(bool v) : kind_(Bool), b_(v) {}
    explicit Json(const std::string& v) : kind_(String), str_(v) {}

    static Json array() { Json j; j.kind_ = Array; return j; }
    static Json object() { Json j; j.kind_ = Object; return j; }

    Kind kind() const { return kind_; }
    bool is_array() const { return kind_ == Array; }
    bool is_object() const { return kind_ == Object; }
    bool is_number() const { return kind_ == Number; }
    bool is_string() const { return kind_ == String; }

    double number() const
    {
        if (kind_ == Number) return num_;
        if (kind_ == Bool) return b_ ? 1.0 : 0.0;
        throw std::runtime_error("JSON value is not a number");
    }
    bool boolean() const
    {
        if (kind_ == Bool) return b_;
        if (kind_ == Number) return num_ != 0.0;
        throw std::runtime_error("JSON value is not a boolean");
    }
    const std::string& string() const
    {
        if (kind_ != String) throw std::runtime_error("JSON value is not a string");
        return str_;
    }
    size_t size() const { return kind_ == Array ? arr_.size() : obj_.size(); }
    const Json& operator[](size_t i) const { return arr_.at(i); }
    Json& at_index(size_t i)
    {
        if (kind_ != Array) { kind_ = Array; arr_.clear(); }
        if (i >= arr_.size()) arr_.resize(i + 1);
        return arr_[i];
    }
    void push_back(const Json& v) { kind_ = Array; arr_.push_back(v); }

    bool contains(const std::string& k) const { return kind_ == Object && obj_.count(k) > 0; }
    const Json& at(const std::string& k) const
    {
        auto it = obj_.find(k);
        if (kind_ != Object || it == obj_.end()) throw std::runtime_error("missing JSON key: " + k);
        return it->second;
    }
    Json& operator[](const std::string& k)
    {
        if (kind_ != Object) { kind_ = Object; obj_.clear(); }
        return obj_[k];
    }
    const std::map<std::string, Json>& items() const { return obj_; }

    static Json parse(const std::string& text)
    {
        size_t p = 0;
        Json v = parse_value(text, p);
        skip(text, p);
        if (p != text.size()) throw std::runtime_error("trailing characters in JSON");
        return v;
    }
    static Json parse_file(const std::string& path)
    {
        std::ifstream in(path);
        if (!in) throw std::runtime_error("cannot open input file " + path);
        std::stringstream ss;
        ss << in.rdbuf();
        return parse(ss.str());
    }

    std::string dump() const
    {
        std::ostringstream o;
        o.precision(17);
        switch (kind_) {
        case Null: o << "null"; break;
        case Bool: o << (b_ ? "true" : "false"); break;
        case Number: o << num_; break;
        case String: o << '"' << str_ << '"'; break;
        case Array:
            o << '[';
            for (size_t i = 0; i < arr_.size(); i++) o << (i ? "," : "") << arr_[i].dump();
            o << ']';
            break;
        case Object: {
            o << '{';
            bool first = true;
            for (auto& kv : obj_) {
                o << (first ? "" : ",") << '"' << kv.first << "\":" << kv.second.dump();
                first = false;
            }
            o << '}';
        }
        }
        return o.str();
    }

  private:
    static void skip(const std::string& t, size_t& p)
    {
        while (p < t.size() && std::isspace((unsigned char)t[p])) p++;
    }
    static Json parse_value(const std::string& t, size_t& p)
    {
        skip(t, p);
        if (p >= t.size()) throw std::runtime_error("unexpected end of JSON");
        const char c = t[p];
        if (c == '{') {
            Json o = object();
            p++;
            skip(t, p);
            if (t[p] == '}') { p++; return o; }
            for (;;) {
                skip(t, p);
                std::string key = parse_string(t, p);
                skip(t, p);
                if (t[p] != ':') throw std::runtime_error("expected ':' in JSON");
                p++;
                o.obj_[key] = parse_value(t, p);
                skip(t, p);
                if (t[p] == ',') { p++; continue; }
                if (t[p] == '}') { p++; return o; }
                throw std::runtime_error("expected ',' or '}' in JSON");
            }
        }
        if (c == '[') {
            Json a = array();
            p++;
            skip(t, p);
            if (t[p] == ']') { p++; return a; }
            for (;;) {
                a.arr_.push_back(parse_value(t, p));
                skip(t, p);
                if (t[p] == ',') { p++; continue; }
                if (t[p] == ']') { p++; return a; }
                throw std::runtime_error("expected ',' or ']' in JSON");
            }
        }
        if (c == '"') return Json(parse_string(t, p));
        if (t.compare(p, 4, "true") == 0) { p += 4; return Json(true); }
        if (t.compare(p, 5, "false") == 0) { p += 5; return Json(false); }
        if (t.compare(p, 4, "null") == 0) { p += 4; return Json(); }
        const char* start = t.c_str() + p;
        char* end = nullptr;
        const double v = std::strtod(start, &end);
        if (end == start) throw std::runtime_error("bad JSON number");
        p += (size_t)(end - start);
        return Json(v);
    }
    static std::string parse_string(const std::string& t, size_t& p)
    {
        if (t[p] != '"') throw std::runtime_error("expected JSON string");
        p++;
        std::string s;
        while (p < t.size() && t[p] != '"') {
            if (t[p] == '\\' && p + 1 < t.size()) p++;
            s += t[p++];
        }
        p++;
        return s;
    }

    Kind kind_ = Null;
    double num_ = 0.0;
    bool b_ = false;
    std::string str_;
    std::vector<Json> arr_;
    std::map<std::string, Json> obj_;
};

}  // namespace cabanapd_shim
