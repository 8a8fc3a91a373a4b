#pragma once
// Strict RFC 8259 JSON document model for scene files.
//
// Behaviour matches the reference loader's contract (include/raytracer/io/json.hpp:26-69,
// src/io/json.cpp:131-307): objects keep insertion order and reject duplicate keys,
// numbers are doubles, nesting is bounded, and every syntax error is reported as
// "JSON parse error at line L, column C: <what>". Serialisation writes the
// shortest round-tripping form of each number.
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>
#include <vector>

namespace rtg {

class JsonValue;
using JsonList = std::vector<JsonValue>;
using JsonMap = std::vector<std::pair<std::string, JsonValue>>;

struct JsonError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class JsonValue {
 public:
  enum class Kind : std::uint8_t { Null, Bool, Number, String, List, Map };

  JsonValue() = default;
  JsonValue(std::nullptr_t) {}
  JsonValue(bool b) : data_(b) {}
  JsonValue(double d) : data_(d) {}
  JsonValue(int i) : data_(double(i)) {}
  JsonValue(std::int64_t i) : data_(double(i)) {}
  JsonValue(std::uint64_t i) : data_(double(i)) {}
  JsonValue(const char* s) : data_(std::string(s)) {}
  JsonValue(std::string s) : data_(std::move(s)) {}
  JsonValue(JsonList l) : data_(std::move(l)) {}
  JsonValue(JsonMap m) : data_(std::move(m)) {}

  Kind kind() const { return static_cast<Kind>(data_.index()); }
  bool is_null() const { return kind() == Kind::Null; }
  bool is_bool() const { return kind() == Kind::Bool; }
  bool is_number() const { return kind() == Kind::Number; }
  bool is_string() const { return kind() == Kind::String; }
  bool is_list() const { return kind() == Kind::List; }
  bool is_map() const { return kind() == Kind::Map; }

  bool boolean() const;
  double number() const;
  const std::string& str() const;
  const JsonList& list() const;
  const JsonMap& map() const;
  JsonList& list();
  JsonMap& map();

  // Lookup in a map; nullptr when absent or when this is not a map.
  const JsonValue* get(const std::string& key) const;
  // Map member access that inserts a null member (turns null into a map).
  JsonValue& operator[](const std::string& key);

  std::string serialize(int indent = 2) const;  // indent < 0: compact
  static JsonValue parse(const std::string& text, int max_depth = 128);

  bool operator==(const JsonValue& o) const { return data_ == o.data_; }

 private:
  std::variant<std::monostate, bool, double, std::string, JsonList, JsonMap> data_;
};

}  // namespace rtg
