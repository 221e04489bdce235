// json_lite.hpp -- a small JSON reader for the solver's input files and the
// material property objects passed through the C ABI.
//
// Supports objects, arrays, numbers, strings (with the common escapes),
// true/false/null.  Numbers are parsed with strtod, so a decimal literal gives
// the same double as any correctly rounded parser.
#pragma once

#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace mpm_b200 {

struct Json {
  enum Type { Null, Bool, Number, String, Array, Object } type = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;  // keeps file order

  bool is_null() const { return type == Null; }
  bool is_object() const { return type == Object; }
  bool is_array() const { return type == Array; }
  bool is_number() const { return type == Number; }
  bool is_bool() const { return type == Bool; }
  bool is_string() const { return type == String; }

  bool contains(const std::string& k) const {
    if (type != Object) return false;
    for (auto& kv : obj)
      if (kv.first == k) return true;
    return false;
  }
  const Json& at(const std::string& k) const {
    if (type != Object) throw std::runtime_error("json: not an object looking up \"" + k + "\"");
    for (auto& kv : obj)
      if (kv.first == k) return kv.second;
    throw std::runtime_error("json: key \"" + k + "\" not found");
  }
  const Json& at(size_t i) const {
    if (type != Array || i >= arr.size()) throw std::runtime_error("json: bad array index");
    return arr[i];
  }
  size_t size() const { return type == Array ? arr.size() : (type == Object ? obj.size() : 0); }
  double as_double() const {
    if (type == Number) return num;
    if (type == Bool) return b ? 1.0 : 0.0;
    throw std::runtime_error("json: value is not a number");
  }
  bool as_bool() const {
    if (type == Bool) return b;
    throw std::runtime_error("json: value is not a boolean");
  }
  const std::string& as_string() const {
    if (type == String) return str;
    throw std::runtime_error("json: value is not a string");
  }
  double get(const std::string& k, double dflt) const {
    return contains(k) ? at(k).as_double() : dflt;
  }
};

class JsonParser {
 public:
  explicit JsonParser(const std::string& s) : s_(s) {}
  Json parse() {
    Json v = value();
    ws();
    if (i_ != s_.size()) fail("trailing characters");
    return v;
  }

 private:
  const std::string& s_;
  size_t i_ = 0;

  [[noreturn]] void fail(const char* what) {
    throw std::runtime_error(std::string("json parse error at offset ") + std::to_string(i_) +
                             ": " + what);
  }
  void ws() {
    while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\n' || s_[i_] == '\t' || s_[i_] == '\r'))
      ++i_;
  }
  bool lit(const char* w) {
    size_t n = 0;
    while (w[n]) ++n;
    if (s_.compare(i_, n, w) == 0) {
      i_ += n;
      return true;
    }
    return false;
  }
  Json value() {
    ws();
    if (i_ >= s_.size()) fail("unexpected end");
    const char c = s_[i_];
    Json v;
    if (c == '{') {
      v.type = Json::Object;
      ++i_;
      ws();
      if (i_ < s_.size() && s_[i_] == '}') {
        ++i_;
        return v;
      }
      while (true) {
        ws();
        if (i_ >= s_.size() || s_[i_] != '"') fail("expected key");
        std::string k = string();
        ws();
        if (i_ >= s_.size() || s_[i_] != ':') fail("expected ':'");
        ++i_;
        v.obj.emplace_back(k, value());
        ws();
        if (i_ < s_.size() && s_[i_] == ',') {
          ++i_;
          continue;
        }
        if (i_ < s_.size() && s_[i_] == '}') {
          ++i_;
          break;
        }
        fail("expected ',' or '}'");
      }
      return v;
    }
    if (c == '[') {
      v.type = Json::Array;
      ++i_;
      ws();
      if (i_ < s_.size() && s_[i_] == ']') {
        ++i_;
        return v;
      }
      while (true) {
        v.arr.push_back(value());
        ws();
        if (i_ < s_.size() && s_[i_] == ',') {
          ++i_;
          continue;
        }
        if (i_ < s_.size() && s_[i_] == ']') {
          ++i_;
          break;
        }
        fail("expected ',' or ']'");
      }
      return v;
    }
    if (c == '"') {
      v.type = Json::String;
      v.str = string();
      return v;
    }
    if (lit("true")) {
      v.type = Json::Bool;
      v.b = true;
      return v;
    }
    if (lit("false")) {
      v.type = Json::Bool;
      v.b = false;
      return v;
    }
    if (lit("null")) return v;
    // number
    const char* begin = s_.c_str() + i_;
    char* end = nullptr;
    const double d = std::strtod(begin, &end);
    if (end == begin) fail("bad value");
    i_ += (size_t)(end - begin);
    v.type = Json::Number;
    v.num = d;
    return v;
  }
  std::string string() {
    std::string out;
    ++i_;  // opening quote
    while (i_ < s_.size() && s_[i_] != '"') {
      char c = s_[i_++];
      if (c == '\\' && i_ < s_.size()) {
        const char e = s_[i_++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (i_ + 4 > s_.size()) fail("bad \\u escape");
            const unsigned cp = (unsigned)std::strtoul(s_.substr(i_, 4).c_str(), nullptr, 16);
            i_ += 4;
            if (cp < 0x80) out += (char)cp;
            else if (cp < 0x800) {
              out += (char)(0xC0 | (cp >> 6));
              out += (char)(0x80 | (cp & 0x3F));
            } else {
              out += (char)(0xE0 | (cp >> 12));
              out += (char)(0x80 | ((cp >> 6) & 0x3F));
              out += (char)(0x80 | (cp & 0x3F));
            }
            break;
          }
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (i_ >= s_.size()) fail("unterminated string");
    ++i_;
    return out;
  }
};

inline Json parse_json(const std::string& s) { return JsonParser(s).parse(); }

}  // namespace mpm_b200
