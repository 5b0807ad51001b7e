#include "json_lite.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

#include "rgpu_internal.h"

namespace rgpu {
namespace {

struct Parser {
  const std::string & s;
  size_t p{0};
  explicit Parser(const std::string & t) : s(t) {}
  [[noreturn]] void fail(const char * what) {
    throw Error(RGPU_ERR_INVALID_ARGUMENT,
                std::string("invalid hypers JSON: ") + what + " at offset " + std::to_string(p));
  }
  void ws() {
    while (p < s.size() && (s[p] == ' ' || s[p] == '\n' || s[p] == '\t' || s[p] == '\r')) ++p;
  }
  bool lit(const char * w) {
    size_t n = std::char_traits<char>::length(w);
    if (s.compare(p, n, w) == 0) {
      p += n;
      return true;
    }
    return false;
  }
  std::string string_body() {
    std::string out;
    ++p;  // opening quote
    while (p < s.size() && s[p] != '"') {
      char c = s[p++];
      if (c == '\\') {
        if (p >= s.size()) fail("bad escape");
        char e = s[p++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u':
            if (p + 4 > s.size()) fail("bad unicode escape");
            out += char(std::strtol(s.substr(p, 4).c_str(), nullptr, 16) & 0x7f);
            p += 4;
            break;
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (p >= s.size()) fail("unterminated string");
    ++p;
    return out;
  }
  Json value() {
    ws();
    if (p >= s.size()) fail("unexpected end");
    Json v;
    char c = s[p];
    if (c == '{') {
      v.type = Json::Object;
      ++p;
      ws();
      if (p < s.size() && s[p] == '}') {
        ++p;
        return v;
      }
      while (true) {
        ws();
        if (p >= s.size() || s[p] != '"') fail("expected key");
        std::string k = string_body();
        ws();
        if (p >= s.size() || s[p] != ':') fail("expected ':'");
        ++p;
        v.obj[k] = value();
        ws();
        if (p < s.size() && s[p] == ',') {
          ++p;
          continue;
        }
        if (p < s.size() && s[p] == '}') {
          ++p;
          break;
        }
        fail("expected ',' or '}'");
      }
    } else if (c == '[') {
      v.type = Json::Array;
      ++p;
      ws();
      if (p < s.size() && s[p] == ']') {
        ++p;
        return v;
      }
      while (true) {
        v.arr.push_back(value());
        ws();
        if (p < s.size() && s[p] == ',') {
          ++p;
          continue;
        }
        if (p < s.size() && s[p] == ']') {
          ++p;
          break;
        }
        fail("expected ',' or ']'");
      }
    } else if (c == '"') {
      v.type = Json::String;
      v.str = string_body();
    } else if (lit("true")) {
      v.type = Json::Bool;
      v.b = true;
    } else if (lit("false")) {
      v.type = Json::Bool;
      v.b = false;
    } else if (lit("null")) {
      v.type = Json::Null;
    } else {
      size_t q = p;
      while (q < s.size() && (std::isdigit((unsigned char)s[q]) || s[q] == '-' || s[q] == '+' ||
                              s[q] == '.' || s[q] == 'e' || s[q] == 'E'))
        ++q;
      if (q == p) fail("unexpected character");
      std::string t = s.substr(p, q - p);
      v.type = Json::Number;
      v.num = std::strtod(t.c_str(), nullptr);
      v.is_int = t.find_first_of(".eE") == std::string::npos;
      p = q;
    }
    return v;
  }
};

void dump_to(const Json & v, std::string & o) {
  switch (v.type) {
    case Json::Null: o += "null"; break;
    case Json::Bool: o += v.b ? "true" : "false"; break;
    case Json::Number: {
      char buf[64];
      if (v.is_int)
        std::snprintf(buf, sizeof buf, "%lld", (long long)v.num);
      else
        std::snprintf(buf, sizeof buf, "%.17g", v.num);
      o += buf;
      break;
    }
    case Json::String: o += '"' + v.str + '"'; break;
    case Json::Array:
      o += '[';
      for (size_t i = 0; i < v.arr.size(); ++i) {
        if (i) o += ',';
        dump_to(v.arr[i], o);
      }
      o += ']';
      break;
    case Json::Object: {
      o += '{';
      bool first = true;
      for (auto & kv : v.obj) {
        if (!first) o += ',';
        first = false;
        o += '"' + kv.first + "\":";
        dump_to(kv.second, o);
      }
      o += '}';
      break;
    }
  }
}

}  // namespace

const Json & Json::at(const std::string & k) const {
  if (type != Object) throw Error(RGPU_ERR_INVALID_ARGUMENT, "hypers: '" + k + "' looked up in a non-object");
  auto it = obj.find(k);
  if (it == obj.end()) throw Error(RGPU_ERR_INVALID_ARGUMENT, "hypers: missing key '" + k + "'");
  return it->second;
}
double Json::as_number() const {
  if (type == Number) return num;
  if (type == Bool) return b ? 1. : 0.;
  throw Error(RGPU_ERR_INVALID_ARGUMENT, "hypers: expected a number");
}
int Json::as_int() const { return int(std::llround(as_number())); }
bool Json::as_bool() const {
  if (type == Bool) return b;
  if (type == Number) return num != 0.;
  throw Error(RGPU_ERR_INVALID_ARGUMENT, "hypers: expected a boolean");
}
const std::string & Json::as_string() const {
  if (type != String) throw Error(RGPU_ERR_INVALID_ARGUMENT, "hypers: expected a string");
  return str;
}
std::string Json::dump() const {
  std::string o;
  dump_to(*this, o);
  return o;
}
Json Json::parse(const std::string & text) {
  Parser p(text);
  Json v = p.value();
  p.ws();
  if (p.p != text.size()) p.fail("trailing characters");
  return v;
}

}  // namespace rgpu
