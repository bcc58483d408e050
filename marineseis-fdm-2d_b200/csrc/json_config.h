// JSON config reader for the reference's model schema (json_template.json).
//
// Path syntax and typing follow the reference's wrapper (include/json_config.hpp
// in the reference: dotted keys with [i] indices, get<int> truncating the
// number like cJSON's valueint, get<float> rounding the double, mismatches
// reported as errors). The parser is a self-contained RFC 8259 reader; no
// cJSON code is used.
#pragma once
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mfdm {

struct JsonValue {
  enum Type { Null, Bool, Number, String, Array, Object } type = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<JsonValue> arr;
  std::vector<std::pair<std::string, JsonValue>> obj;
};

class JsonError : public std::runtime_error {
 public:
  explicit JsonError(const std::string& m) : std::runtime_error(m) {}
};

class JsonConfig {
 public:
  static JsonConfig from_file(const std::string& path);
  static JsonConfig from_text(const std::string& text, const std::string& name = "<text>");

  bool has(const std::string& path) const { return find(path) != nullptr; }
  int get_int(const std::string& path) const;
  float get_float(const std::string& path) const;
  std::string get_string(const std::string& path) const;
  size_t size(const std::string& path) const;
  int get_int(const std::string& path, size_t index) const;

 private:
  JsonValue root_;
  std::string name_;
  const JsonValue* find(const std::string& path) const;
  const JsonValue& need(const std::string& path) const;
};

}  // namespace mfdm
