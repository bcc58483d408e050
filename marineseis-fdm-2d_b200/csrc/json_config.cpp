#include "json_config.h"

#include <cerrno>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace mfdm {
namespace {

struct Parser {
  const char* p;
  const char* begin;
  std::string name;

  [[noreturn]] void fail(const char* what) const {
    std::ostringstream os;
    os << "Failed to parse JSON file: " << name << " (" << what << " at byte " << (p - begin)
       << ")";
    throw JsonError(os.str());
  }
  void ws() {
    while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r') ++p;
  }
  static int hex(char c) {
    if (c >= '0' && c <= '9') return c - '0';
    if (c >= 'a' && c <= 'f') return c - 'a' + 10;
    if (c >= 'A' && c <= 'F') return c - 'A' + 10;
    return -1;
  }
  std::string string_lit() {
    if (*p != '"') fail("expected string");
    ++p;
    std::string out;
    while (*p && *p != '"') {
      if (*p != '\\') {
        out.push_back(*p++);
        continue;
      }
      ++p;
      switch (*p) {
        case '"': out.push_back('"'); break;
        case '\\': out.push_back('\\'); break;
        case '/': out.push_back('/'); break;
        case 'b': out.push_back('\b'); break;
        case 'f': out.push_back('\f'); break;
        case 'n': out.push_back('\n'); break;
        case 'r': out.push_back('\r'); break;
        case 't': out.push_back('\t'); break;
        case 'u': {
          unsigned cp = 0;
          for (int k = 1; k <= 4; ++k) {
            const int h = hex(p[k]);
            if (h < 0) fail("bad \\u escape");
            cp = cp * 16 + unsigned(h);
          }
          p += 4;
          if (cp < 0x80) {
            out.push_back(char(cp));
          } else if (cp < 0x800) {
            out.push_back(char(0xC0 | (cp >> 6)));
            out.push_back(char(0x80 | (cp & 0x3F)));
          } else {
            out.push_back(char(0xE0 | (cp >> 12)));
            out.push_back(char(0x80 | ((cp >> 6) & 0x3F)));
            out.push_back(char(0x80 | (cp & 0x3F)));
          }
          break;
        }
        default: fail("bad escape");
      }
      ++p;
    }
    if (*p != '"') fail("unterminated string");
    ++p;
    return out;
  }
  JsonValue value(int depth) {
    if (depth > 512) fail("nesting too deep");
    ws();
    JsonValue v;
    if (*p == '{') {
      v.type = JsonValue::Object;
      ++p;
      ws();
      if (*p == '}') { ++p; return v; }
      for (;;) {
        ws();
        std::string key = string_lit();
        ws();
        if (*p != ':') fail("expected ':'");
        ++p;
        v.obj.emplace_back(std::move(key), value(depth + 1));
        ws();
        if (*p == ',') { ++p; continue; }
        if (*p == '}') { ++p; return v; }
        fail("expected ',' or '}'");
      }
    }
    if (*p == '[') {
      v.type = JsonValue::Array;
      ++p;
      ws();
      if (*p == ']') { ++p; return v; }
      for (;;) {
        v.arr.push_back(value(depth + 1));
        ws();
        if (*p == ',') { ++p; continue; }
        if (*p == ']') { ++p; return v; }
        fail("expected ',' or ']'");
      }
    }
    if (*p == '"') {
      v.type = JsonValue::String;
      v.str = string_lit();
      return v;
    }
    if (!std::strncmp(p, "true", 4)) { p += 4; v.type = JsonValue::Bool; v.b = true; return v; }
    if (!std::strncmp(p, "false", 5)) { p += 5; v.type = JsonValue::Bool; return v; }
    if (!std::strncmp(p, "null", 4)) { p += 4; return v; }
    if (*p == '-' || (*p >= '0' && *p <= '9')) {
      char* end = nullptr;
      v.num = std::strtod(p, &end);
      if (end == p) fail("bad number");
      v.type = JsonValue::Number;
      p = end;
      return v;
    }
    fail("unexpected character");
  }
};

std::string quote(const std::string& s) { return "'" + s + "'"; }

}  // namespace

JsonConfig JsonConfig::from_text(const std::string& text, const std::string& name) {
  if (text.empty()) throw JsonError("JSON file is empty: " + name);
  Parser ps{text.c_str(), text.c_str(), name};
  JsonConfig c;
  c.root_ = ps.value(0);
  ps.ws();
  if (*ps.p != '\0') ps.fail("trailing characters");
  c.name_ = name;
  return c;
}

JsonConfig JsonConfig::from_file(const std::string& path) {
  std::ifstream f(path);
  if (!f.is_open()) throw JsonError("Cannot open JSON file: " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return from_text(ss.str(), path);
}

// Dotted path walk with [i] indices (reference include/json_config.hpp:241-356).
const JsonValue* JsonConfig::find(const std::string& path) const {
  const JsonValue* cur = &root_;
  size_t pos = 0;
  while (pos < path.size()) {
    if (path[pos] == '.') { ++pos; continue; }
    if (path[pos] != '[') {
      const size_t b = pos;
      while (pos < path.size() && path[pos] != '.' && path[pos] != '[') ++pos;
      const std::string key = path.substr(b, pos - b);
      if (cur->type != JsonValue::Object) return nullptr;
      const JsonValue* next = nullptr;
      for (const auto& kv : cur->obj)
        if (kv.first == key) { next = &kv.second; break; }
      if (!next) return nullptr;
      cur = next;
    }
    while (pos < path.size() && path[pos] == '[') {
      const size_t close = path.find(']', pos);
      if (close == std::string::npos || close == pos + 1) return nullptr;
      const std::string idx = path.substr(pos + 1, close - pos - 1);
      char* end = nullptr;
      const long i = std::strtol(idx.c_str(), &end, 10);
      if (end == idx.c_str() || *end != '\0' || i < 0) return nullptr;
      if (cur->type != JsonValue::Array || size_t(i) >= cur->arr.size()) return nullptr;
      cur = &cur->arr[size_t(i)];
      pos = close + 1;
    }
  }
  return cur;
}

const JsonValue& JsonConfig::need(const std::string& path) const {
  const JsonValue* v = find(path);
  if (!v) throw JsonError("JSON path not found: " + path);
  return *v;
}

static int to_int(const JsonValue& v, const std::string& path) {
  if (v.type != JsonValue::Number)
    throw JsonError("JSON type mismatch at " + quote(path) + ": expected int");
  if (v.num >= double(INT_MAX)) return INT_MAX;
  if (v.num <= double(INT_MIN)) return INT_MIN;
  return int(v.num);
}

int JsonConfig::get_int(const std::string& path) const { return to_int(need(path), path); }

float JsonConfig::get_float(const std::string& path) const {
  const JsonValue& v = need(path);
  if (v.type != JsonValue::Number)
    throw JsonError("JSON type mismatch at " + quote(path) + ": expected float");
  return float(v.num);
}

std::string JsonConfig::get_string(const std::string& path) const {
  const JsonValue& v = need(path);
  if (v.type != JsonValue::String)
    throw JsonError("JSON type mismatch at " + quote(path) + ": expected string");
  return v.str;
}

size_t JsonConfig::size(const std::string& path) const {
  const JsonValue& v = need(path);
  if (v.type != JsonValue::Array) throw JsonError("JSON node is not an array: " + path);
  return v.arr.size();
}

int JsonConfig::get_int(const std::string& path, size_t index) const {
  const JsonValue& v = need(path);
  if (v.type != JsonValue::Array) throw JsonError("JSON node is not an array: " + path);
  if (index >= v.arr.size())
    throw JsonError("Array index out of range: " + path + "[" + std::to_string(index) + "]");
  return to_int(v.arr[index], path + "[" + std::to_string(index) + "]");
}

}  // namespace mfdm
