// Minimal JSON (see json.h).
#include "json.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <fstream>
#include <sstream>

#include "runtime.h"

namespace r2 {

namespace {
const Json& null_json() {
  static const Json n;
  return n;
}

struct Parser {
  const std::string& s;
  size_t i = 0;
  explicit Parser(const std::string& t) : s(t) {}

  [[noreturn]] void fail(const std::string& what) {
    throw Error{R2_ERR_INVALID_CONFIG, "JSON parse error at offset " + std::to_string(i) + ": " + what};
  }
  void skip() {
    for (;;) {
      while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
      if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/') {
        while (i < s.size() && s[i] != '\n') ++i;
        continue;
      }
      if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*') {
        size_t e = s.find("*/", i + 2);
        if (e == std::string::npos) fail("unterminated comment");
        i = e + 2;
        continue;
      }
      break;
    }
  }
  Json value() {
    skip();
    if (i >= s.size()) fail("unexpected end");
    char c = s[i];
    if (c == '{') return object();
    if (c == '[') return array();
    if (c == '"') return Json::string(str());
    if (s.compare(i, 4, "true") == 0) { i += 4; return Json::boolean(true); }
    if (s.compare(i, 5, "false") == 0) { i += 5; return Json::boolean(false); }
    if (s.compare(i, 4, "null") == 0) { i += 4; return Json(); }
    if (c == '-' || c == '+' || c == '.' || (c >= '0' && c <= '9')) {
      const char* b = s.c_str() + i;
      char* e = nullptr;
      double v = strtod(b, &e);
      if (e == b) fail("bad number");
      i += (size_t)(e - b);
      return Json::number(v);
    }
    fail(std::string("unexpected character '") + c + "'");
  }
  std::string str() {
    ++i;  // opening quote
    std::string out;
    while (i < s.size() && s[i] != '"') {
      char c = s[i++];
      if (c == '\\') {
        if (i >= s.size()) fail("bad escape");
        char e = s[i++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (i + 4 > s.size()) fail("bad unicode escape");
            unsigned cp = (unsigned)strtoul(s.substr(i, 4).c_str(), nullptr, 16);
            i += 4;
            if (cp < 0x80) out += (char)cp;
            else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
            else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
            break;
          }
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (i >= s.size()) fail("unterminated string");
    ++i;
    return out;
  }
  Json array() {
    ++i;
    Json a = Json::array();
    skip();
    if (i < s.size() && s[i] == ']') { ++i; return a; }
    for (;;) {
      a.push(value());
      skip();
      if (i < s.size() && s[i] == ',') { ++i; skip(); if (i < s.size() && s[i] == ']') { ++i; return a; } continue; }
      if (i < s.size() && s[i] == ']') { ++i; return a; }
      fail("expected ',' or ']'");
    }
  }
  Json object() {
    ++i;
    Json o = Json::object();
    skip();
    if (i < s.size() && s[i] == '}') { ++i; return o; }
    for (;;) {
      skip();
      if (i >= s.size() || s[i] != '"') fail("expected key");
      std::string k = str();
      skip();
      if (i >= s.size() || s[i] != ':') fail("expected ':'");
      ++i;
      o.set(k, value());
      skip();
      if (i < s.size() && s[i] == ',') { ++i; skip(); if (i < s.size() && s[i] == '}') { ++i; return o; } continue; }
      if (i < s.size() && s[i] == '}') { ++i; return o; }
      fail("expected ',' or '}'");
    }
  }
};

void dump_string(std::string& out, const std::string& s) {
  out += '"';
  for (char c : s) {
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\n': out += "\\n"; break;
      case '\t': out += "\\t"; break;
      case '\r': out += "\\r"; break;
      default: out += c;
    }
  }
  out += '"';
}
}  // namespace

double Json::as_number() const {
  if (type_ == Number) return num_;
  if (type_ == Bool) return b_ ? 1.0 : 0.0;
  throw Error{R2_ERR_INVALID_CONFIG, "JSON value is not a number"};
}
bool Json::as_bool() const {
  if (type_ == Bool) return b_;
  if (type_ == Number) return num_ != 0.0;
  throw Error{R2_ERR_INVALID_CONFIG, "JSON value is not a boolean"};
}
const std::string& Json::as_string() const {
  if (type_ != String) throw Error{R2_ERR_INVALID_CONFIG, "JSON value is not a string"};
  return str_;
}
const Json& Json::operator[](size_t i) const {
  if (type_ != Array || i >= arr_.size()) return null_json();
  return arr_[i];
}
const Json& Json::operator[](const std::string& key) const {
  if (type_ != Object) return null_json();
  auto it = obj_.find(key);
  return it == obj_.end() ? null_json() : it->second;
}
Json& Json::set(const std::string& key, Json v) {
  if (type_ == Null) type_ = Object;
  obj_[key] = std::move(v);
  return obj_[key];
}
Json& Json::push(Json v) {
  if (type_ == Null) type_ = Array;
  arr_.push_back(std::move(v));
  return arr_.back();
}

Json Json::parse(const std::string& text) {
  Parser p(text);
  Json v = p.value();
  p.skip();
  if (p.i != text.size()) p.fail("trailing characters");
  return v;
}

void Json::dump_to(std::string& out, int indent, int depth) const {
  auto nl = [&](int d) {
    out += '\n';
    out.append((size_t)(indent * d), ' ');
  };
  switch (type_) {
    case Null: out += "null"; break;
    case Bool: out += b_ ? "true" : "false"; break;
    case Number: {
      char b[40];
      if (num_ == floor(num_) && fabs(num_) < 1e15) snprintf(b, sizeof(b), "%.1f", num_);
      else snprintf(b, sizeof(b), "%.17g", num_);
      // integers stay integers
      if (num_ == floor(num_) && fabs(num_) < 1e15) snprintf(b, sizeof(b), "%lld", (long long)num_);
      out += b;
      break;
    }
    case String: dump_string(out, str_); break;
    case Array:
      if (arr_.empty()) { out += "[]"; break; }
      out += '[';
      for (size_t k = 0; k < arr_.size(); ++k) {
        if (k) out += ',';
        nl(depth + 1);
        arr_[k].dump_to(out, indent, depth + 1);
      }
      nl(depth);
      out += ']';
      break;
    case Object:
      if (obj_.empty()) { out += "{}"; break; }
      out += '{';
      {
        bool first = true;
        for (const auto& kv : obj_) {
          if (!first) out += ',';
          first = false;
          nl(depth + 1);
          dump_string(out, kv.first);
          out += ": ";
          kv.second.dump_to(out, indent, depth + 1);
        }
      }
      nl(depth);
      out += '}';
      break;
  }
}

std::string Json::dump(int indent) const {
  std::string out;
  dump_to(out, indent, 0);
  return out;
}

std::string read_text_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error{R2_ERR_IO, "cannot open " + path};
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

}  // namespace r2
