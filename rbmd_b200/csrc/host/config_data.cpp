// config_data.cpp -- a small recursive-descent JSON parser for ConfigData.
#include "config_data.h"

#include <cctype>
#include <cstdlib>

namespace rbx_host {
namespace {

struct Parser {
  const std::string& s;
  size_t i = 0;
  explicit Parser(const std::string& t) : s(t) {}

  [[noreturn]] void Fail(const char* what) {
    throw std::runtime_error(std::string("JSON parse error at offset ") + std::to_string(i) +
                             ": " + what);
  }
  // Whitespace and comments: "// ..." to the end of the line, "/* ... */".
  void Ws() {
    for (;;) {
      while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
      if (i + 1 >= s.size() || s[i] != '/') return;
      if (s[i + 1] == '/') {
        while (i < s.size() && s[i] != '\n') ++i;
      } else if (s[i + 1] == '*') {
        const size_t end = s.find("*/", i + 2);
        if (end == std::string::npos) Fail("unterminated comment");
        i = end + 2;
      } else {
        return;
      }
    }
  }
  bool Eat(char c) {
    Ws();
    if (i < s.size() && s[i] == c) {
      ++i;
      return true;
    }
    return false;
  }
  void Expect(char c) {
    if (!Eat(c)) Fail("unexpected character");
  }
  std::string Str() {
    Expect('"');
    std::string out;
    while (i < s.size() && s[i] != '"') {
      char c = s[i++];
      if (c == '\\') {
        if (i >= s.size()) Fail("bad escape");
        const char e = s[i++];
        switch (e) {
          case '"': out += '"'; break;
          case '\\': out += '\\'; break;
          case '/': out += '/'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'n': out += '\n'; break;
          case 'r': out += '\r'; break;
          case 't': out += '\t'; break;
          case 'u': {
            if (i + 4 > s.size()) Fail("bad \\u escape");
            const unsigned cp = (unsigned)std::strtoul(s.substr(i, 4).c_str(), nullptr, 16);
            i += 4;
            if (cp < 0x80) {
              out += (char)cp;
            } else if (cp < 0x800) {
              out += (char)(0xC0 | (cp >> 6));
              out += (char)(0x80 | (cp & 0x3F));
            } else {
              out += (char)(0xE0 | (cp >> 12));
              out += (char)(0x80 | ((cp >> 6) & 0x3F));
              out += (char)(0x80 | (cp & 0x3F));
            }
            break;
          }
          default: Fail("bad escape");
        }
      } else {
        out += c;
      }
    }
    if (i >= s.size()) Fail("unterminated string");
    ++i;
    return out;
  }
  JsonValue Value() {
    Ws();
    if (i >= s.size()) Fail("unexpected end");
    JsonValue v;
    const char c = s[i];
    if (c == '{') {
      ++i;
      v.kind = JsonValue::Object;
      if (Eat('}')) return v;
      do {
        Ws();
        std::string k = Str();
        Expect(':');
        v.obj[k] = Value();
      } while (Eat(','));
      Expect('}');
    } else if (c == '[') {
      ++i;
      v.kind = JsonValue::Array;
      if (Eat(']')) return v;
      do {
        v.arr.push_back(Value());
      } while (Eat(','));
      Expect(']');
    } else if (c == '"') {
      v.kind = JsonValue::String;
      v.str = Str();
    } else if (s.compare(i, 4, "true") == 0) {
      i += 4;
      v.kind = JsonValue::Bool;
      v.b = true;
    } else if (s.compare(i, 5, "false") == 0) {
      i += 5;
      v.kind = JsonValue::Bool;
    } else if (s.compare(i, 4, "null") == 0) {
      i += 4;
    } else {
      char* end = nullptr;
      v.num = std::strtod(s.c_str() + i, &end);
      if (end == s.c_str() + i) Fail("bad value");
      i = (size_t)(end - s.c_str());
      v.kind = JsonValue::Number;
    }
    return v;
  }
};

}  // namespace

JsonValue ParseJson(const std::string& text) {
  Parser p(text);
  if (text.compare(0, 3, "\xEF\xBB\xBF") == 0) p.i = 3;  // UTF-8 byte-order mark
  JsonValue v = p.Value();
  p.Ws();
  if (p.i != text.size()) p.Fail("trailing characters");
  return v;
}

}  // namespace rbx_host
