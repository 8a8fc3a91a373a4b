#include "host/json.hpp"

#include <charconv>
#include <cmath>
#include <cstdio>
#include <string_view>

namespace rtg {

namespace {

const char* kind_name(JsonValue::Kind k) {
  static const char* names[] = {"null", "bool", "number", "string", "array", "object"};
  return names[static_cast<int>(k)];
}

[[noreturn]] void wrong_kind(const char* want, JsonValue::Kind got) {
  throw JsonError(std::string("expected ") + want + ", got " + kind_name(got));
}

}  // namespace

bool JsonValue::boolean() const {
  if (auto* p = std::get_if<bool>(&data_)) return *p;
  wrong_kind("bool", kind());
}
double JsonValue::number() const {
  if (auto* p = std::get_if<double>(&data_)) return *p;
  wrong_kind("number", kind());
}
const std::string& JsonValue::str() const {
  if (auto* p = std::get_if<std::string>(&data_)) return *p;
  wrong_kind("string", kind());
}
const JsonList& JsonValue::list() const {
  if (auto* p = std::get_if<JsonList>(&data_)) return *p;
  wrong_kind("array", kind());
}
const JsonMap& JsonValue::map() const {
  if (auto* p = std::get_if<JsonMap>(&data_)) return *p;
  wrong_kind("object", kind());
}
JsonList& JsonValue::list() {
  if (auto* p = std::get_if<JsonList>(&data_)) return *p;
  wrong_kind("array", kind());
}
JsonMap& JsonValue::map() {
  if (auto* p = std::get_if<JsonMap>(&data_)) return *p;
  wrong_kind("object", kind());
}

const JsonValue* JsonValue::get(const std::string& key) const {
  const auto* m = std::get_if<JsonMap>(&data_);
  if (!m) return nullptr;
  for (const auto& kv : *m)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

JsonValue& JsonValue::operator[](const std::string& key) {
  if (is_null()) data_ = JsonMap{};
  JsonMap& m = map();
  for (auto& kv : m)
    if (kv.first == key) return kv.second;
  m.emplace_back(key, JsonValue{});
  return m.back().second;
}

// ---------------------------------------------------------------------------
// Writer
namespace {

void put_string(std::string& out, const std::string& s) {
  out.push_back('"');
  for (const unsigned char c : s) {
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\b': out += "\\b"; break;
      case '\f': out += "\\f"; break;
      case '\n': out += "\\n"; break;
      case '\r': out += "\\r"; break;
      case '\t': out += "\\t"; break;
      default:
        if (c < 0x20) {
          char esc[8];
          std::snprintf(esc, sizeof esc, "\\u%04x", unsigned(c));
          out += esc;
        } else {
          out.push_back(static_cast<char>(c));
        }
    }
  }
  out.push_back('"');
}

void put_number(std::string& out, double d) {
  if (!std::isfinite(d)) { out += "null"; return; }
  char buf[40];
  const auto res = std::to_chars(buf, buf + sizeof buf, d);  // shortest round trip
  out.append(buf, res.ptr);
}

void put_value(std::string& out, const JsonValue& v, int indent, int depth) {
  const bool pretty = indent >= 0;
  auto line = [&](int d) {
    if (!pretty) return;
    out.push_back('\n');
    out.append(static_cast<std::size_t>(indent) * static_cast<std::size_t>(d), ' ');
  };
  switch (v.kind()) {
    case JsonValue::Kind::Null: out += "null"; return;
    case JsonValue::Kind::Bool: out += v.boolean() ? "true" : "false"; return;
    case JsonValue::Kind::Number: put_number(out, v.number()); return;
    case JsonValue::Kind::String: put_string(out, v.str()); return;
    case JsonValue::Kind::List: {
      const JsonList& l = v.list();
      // Vectors and colours (short lists of scalars) stay on one line.
      bool inline_list = l.size() <= 4;
      for (const auto& e : l) inline_list = inline_list && !e.is_list() && !e.is_map() && !e.is_string();
      out.push_back('[');
      for (std::size_t i = 0; i < l.size(); ++i) {
        if (i) out += (pretty && inline_list) ? ", " : ",";
        if (!inline_list) line(depth + 1);
        put_value(out, l[i], indent, depth + 1);
      }
      if (!inline_list && !l.empty()) line(depth);
      out.push_back(']');
      return;
    }
    case JsonValue::Kind::Map: {
      const JsonMap& m = v.map();
      out.push_back('{');
      for (std::size_t i = 0; i < m.size(); ++i) {
        if (i) out.push_back(',');
        line(depth + 1);
        put_string(out, m[i].first);
        out += pretty ? ": " : ":";
        put_value(out, m[i].second, indent, depth + 1);
      }
      if (!m.empty()) line(depth);
      out.push_back('}');
      return;
    }
  }
}

// ---------------------------------------------------------------------------
// Reader: recursive descent with a nesting bound.
class Reader {
 public:
  Reader(const std::string& text, int max_depth) : s_(text), limit_(max_depth) {}

  JsonValue document() {
    JsonValue v = value(0);
    blank();
    if (at_ != s_.size()) error("trailing characters after JSON value");
    return v;
  }

 private:
  [[noreturn]] void error(const std::string& what) const {
    std::size_t line = 1, col = 1;
    for (std::size_t i = 0; i < at_ && i < s_.size(); ++i) {
      if (s_[i] == '\n') { ++line; col = 1; }
      else ++col;
    }
    throw JsonError("JSON parse error at line " + std::to_string(line) + ", column " + std::to_string(col) + ": " +
                    what);
  }
  char cur() const { return at_ < s_.size() ? s_[at_] : '\0'; }
  bool digit() const { return cur() >= '0' && cur() <= '9'; }
  void blank() {
    while (at_ < s_.size()) {
      const char c = s_[at_];
      if (c != ' ' && c != '\t' && c != '\n' && c != '\r') break;
      ++at_;
    }
  }
  void need(char c) {
    if (cur() != c) error(std::string("expected '") + c + "'");
    ++at_;
  }
  bool word(std::string_view w) {
    if (s_.compare(at_, w.size(), w) != 0) return false;
    at_ += w.size();
    return true;
  }

  JsonValue value(int depth) {
    if (depth > limit_) error("nesting too deep");
    blank();
    const char c = cur();
    switch (c) {
      case '{': return object(depth);
      case '[': return array(depth);
      case '"': return JsonValue(string());
      default: break;
    }
    if (c == '-' || (c >= '0' && c <= '9')) return JsonValue(number());
    if (word("true")) return JsonValue(true);
    if (word("false")) return JsonValue(false);
    if (word("null")) return JsonValue(nullptr);
    if (c == '\0') error("unexpected end of input");
    error(std::string("unexpected character '") + c + "'");
  }

  JsonValue object(int depth) {
    need('{');
    JsonMap m;
    blank();
    if (cur() == '}') { ++at_; return JsonValue(std::move(m)); }
    while (true) {
      blank();
      if (cur() != '"') error("expected string key");
      std::string key = string();
      for (const auto& kv : m)
        if (kv.first == key) error("duplicate key '" + key + "'");
      blank();
      need(':');
      JsonValue v = value(depth + 1);
      m.emplace_back(std::move(key), std::move(v));
      blank();
      if (cur() == ',') { ++at_; continue; }
      need('}');
      return JsonValue(std::move(m));
    }
  }

  JsonValue array(int depth) {
    need('[');
    JsonList l;
    blank();
    if (cur() == ']') { ++at_; return JsonValue(std::move(l)); }
    while (true) {
      l.push_back(value(depth + 1));
      blank();
      if (cur() == ',') { ++at_; continue; }
      need(']');
      return JsonValue(std::move(l));
    }
  }

  unsigned hex4() {
    if (at_ + 4 > s_.size()) error("truncated \\u escape");
    unsigned v = 0;
    for (int k = 0; k < 4; ++k) {
      const char h = s_[at_++];
      unsigned d;
      if (h >= '0' && h <= '9') d = unsigned(h - '0');
      else if (h >= 'a' && h <= 'f') d = unsigned(h - 'a') + 10;
      else if (h >= 'A' && h <= 'F') d = unsigned(h - 'A') + 10;
      else error("bad hex digit in \\u escape");
      v = (v << 4) | d;
    }
    return v;
  }

  static void utf8(std::string& out, unsigned cp) {
    if (cp <= 0x7F) {
      out.push_back(char(cp));
    } else if (cp <= 0x7FF) {
      out.push_back(char(0xC0 | (cp >> 6)));
      out.push_back(char(0x80 | (cp & 0x3F)));
    } else if (cp <= 0xFFFF) {
      out.push_back(char(0xE0 | (cp >> 12)));
      out.push_back(char(0x80 | ((cp >> 6) & 0x3F)));
      out.push_back(char(0x80 | (cp & 0x3F)));
    } else {
      out.push_back(char(0xF0 | (cp >> 18)));
      out.push_back(char(0x80 | ((cp >> 12) & 0x3F)));
      out.push_back(char(0x80 | ((cp >> 6) & 0x3F)));
      out.push_back(char(0x80 | (cp & 0x3F)));
    }
  }

  std::string string() {
    need('"');
    std::string out;
    while (true) {
      if (at_ >= s_.size()) error("unterminated string");
      const char c = s_[at_++];
      if (c == '"') return out;
      if (static_cast<unsigned char>(c) < 0x20) error("control character in string");
      if (c != '\\') { out.push_back(c); continue; }
      if (at_ >= s_.size()) error("unterminated escape");
      const char e = s_[at_++];
      switch (e) {
        case '"': case '\\': case '/': out.push_back(e); break;
        case 'b': out.push_back('\b'); break;
        case 'f': out.push_back('\f'); break;
        case 'n': out.push_back('\n'); break;
        case 'r': out.push_back('\r'); break;
        case 't': out.push_back('\t'); break;
        case 'u': {
          unsigned cp = hex4();
          if (cp >= 0xDC00 && cp <= 0xDFFF) error("unpaired surrogate");
          if (cp >= 0xD800 && cp <= 0xDBFF) {
            if (!word("\\u")) error("unpaired surrogate");
            const unsigned low = hex4();
            if (low < 0xDC00 || low > 0xDFFF) error("invalid low surrogate");
            cp = 0x10000 + ((cp - 0xD800) << 10) + (low - 0xDC00);
          }
          utf8(out, cp);
          break;
        }
        default: error("invalid escape");
      }
    }
  }

  double number() {
    const std::size_t begin = at_;
    if (cur() == '-') ++at_;
    if (cur() == '0') {
      ++at_;
    } else if (digit()) {
      while (digit()) ++at_;
    } else {
      error("invalid number");
    }
    if (cur() == '.') {
      ++at_;
      if (!digit()) error("digit expected after '.'");
      while (digit()) ++at_;
    }
    if (cur() == 'e' || cur() == 'E') {
      ++at_;
      if (cur() == '+' || cur() == '-') ++at_;
      if (!digit()) error("digit expected in exponent");
      while (digit()) ++at_;
    }
    double d = 0;
    const char* first = s_.data() + begin;
    const char* last = s_.data() + at_;
    const auto res = std::from_chars(first, last, d);
    if (res.ec != std::errc() || res.ptr != last || !std::isfinite(d)) error("number out of range");
    return d;
  }

  const std::string& s_;
  std::size_t at_ = 0;
  int limit_;
};

}  // namespace

std::string JsonValue::serialize(int indent) const {
  std::string out;
  put_value(out, *this, indent, 0);
  return out;
}

JsonValue JsonValue::parse(const std::string& text, int max_depth) { return Reader(text, max_depth).document(); }

}  // namespace rtg
