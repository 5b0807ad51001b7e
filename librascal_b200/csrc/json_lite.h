// Minimal JSON value and parser for calculator hypers.
//
// The reference passes hypers as a JSON document (nlohmann::json built from
// the Python dict, bindings/bind_py_representation_calculator.cc:43-47). This
// is a small self-contained reader for that document: objects, arrays,
// strings, numbers, booleans and null. `dump()` writes a canonical compact
// form (keys sorted, as nlohmann::json's std::map storage does) used for the
// calculator name.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace rgpu {

struct Json {
  enum Type { Null, Bool, Number, String, Array, Object } type{Null};
  bool b{false};
  double num{0.};
  bool is_int{false};
  std::string str;
  std::vector<Json> arr;
  std::map<std::string, Json> obj;

  bool has(const std::string & k) const { return type == Object && obj.count(k); }
  const Json & at(const std::string & k) const;
  double as_number() const;
  int as_int() const;
  bool as_bool() const;
  const std::string & as_string() const;
  std::string dump() const;

  static Json parse(const std::string & text);
};

}  // namespace rgpu
