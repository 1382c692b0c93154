// Minimal JSON value with a parser that accepts // and /* */ comments (the
// reference parses config.json and scenedescription.json with comments
// ignored, raytracer/src/backend/config_loader.cu:325,356) and a serializer
// with sorted object keys and two-space indentation (nlohmann's dump(2)).
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace r2 {

class Json {
 public:
  enum Type { Null, Bool, Number, String, Array, Object };
  Json() = default;
  static Json number(double v) { Json j; j.type_ = Number; j.num_ = v; return j; }
  static Json boolean(bool v) { Json j; j.type_ = Bool; j.b_ = v; return j; }
  static Json string(const std::string& s) { Json j; j.type_ = String; j.str_ = s; return j; }
  static Json array() { Json j; j.type_ = Array; return j; }
  static Json object() { Json j; j.type_ = Object; return j; }

  Type type() const { return type_; }
  bool is_null() const { return type_ == Null; }
  bool is_number() const { return type_ == Number; }
  bool is_string() const { return type_ == String; }
  bool is_array() const { return type_ == Array; }
  bool is_object() const { return type_ == Object; }
  bool is_bool() const { return type_ == Bool; }

  double as_number() const;
  bool as_bool() const;
  const std::string& as_string() const;
  size_t size() const { return type_ == Array ? arr_.size() : (type_ == Object ? obj_.size() : 0); }
  const Json& operator[](size_t i) const;
  Json& at(size_t i) { return arr_.at(i); }
  // Object member; a missing member reads as null (like nlohmann's const access).
  const Json& operator[](const std::string& key) const;
  bool has(const std::string& key) const { return type_ == Object && obj_.count(key) > 0; }
  Json& set(const std::string& key, Json v);
  Json& push(Json v);
  const std::map<std::string, Json>& items() const { return obj_; }
  const std::vector<Json>& elements() const { return arr_; }

  static Json parse(const std::string& text);  // throws r2::Error(R2_ERR_INVALID_CONFIG)
  std::string dump(int indent = 2) const;

 private:
  Type type_ = Null;
  bool b_ = false;
  double num_ = 0.0;
  std::string str_;
  std::vector<Json> arr_;
  std::map<std::string, Json> obj_;
  void dump_to(std::string& out, int indent, int depth) const;
};

std::string read_text_file(const std::string& path);  // throws R2_ERR_IO

}  // namespace r2
