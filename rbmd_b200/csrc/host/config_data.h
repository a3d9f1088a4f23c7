// config_data.h -- JSON configuration reader with the lookup interface of
// RBMD's ConfigData (src/data_manager/include/config_data.h:53-159):
// Get<T>(key, path...), GetArray<T>(key, path...), PathExists({path...}).
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace rbx_host {

struct JsonValue {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<JsonValue> arr;
  std::map<std::string, JsonValue> obj;
};

// Parses RFC 8259 JSON plus // and /* */ comments and a leading UTF-8
// byte-order mark, as ConfigData::ParseJsonFile reads the reference's config
// files (nlohmann::ordered_json::parse with ignore_comments, config_data.h:239-256).
// Throws std::runtime_error on bad input.
JsonValue ParseJson(const std::string& text);

class ConfigData {
 public:
  explicit ConfigData(const std::string& json_text) : _root(ParseJson(json_text)) {}

  bool PathExists(const std::vector<std::string>& path) const { return Find(path) != nullptr; }

  template <typename T, typename... Path>
  T Get(const std::string& key, const Path&... path) const {
    std::vector<std::string> p{path..., key};
    const JsonValue* v = Find(p);
    if (!v) throw std::runtime_error("missing JSON key: " + Join(p));
    return Convert<T>(*v, Join(p));
  }

  template <typename T, typename... Path>
  std::vector<T> GetArray(const std::string& key, const Path&... path) const {
    std::vector<std::string> p{path..., key};
    const JsonValue* v = Find(p);
    if (!v || v->kind != JsonValue::Array) throw std::runtime_error("missing JSON array: " + Join(p));
    std::vector<T> out;
    for (const auto& e : v->arr) out.push_back(Convert<T>(e, Join(p)));
    return out;
  }

 private:
  const JsonValue* Find(const std::vector<std::string>& path) const {
    const JsonValue* cur = &_root;
    for (const auto& k : path) {
      if (cur->kind != JsonValue::Object) return nullptr;
      auto it = cur->obj.find(k);
      if (it == cur->obj.end()) return nullptr;
      cur = &it->second;
    }
    return cur;
  }
  static std::string Join(const std::vector<std::string>& p) {
    std::string s;
    for (size_t i = 0; i < p.size(); ++i) s += (i ? "." : "") + p[i];
    return s;
  }
  template <typename T>
  static T Convert(const JsonValue& v, const std::string& where);

  JsonValue _root;
};

template <>
inline double ConfigData::Convert<double>(const JsonValue& v, const std::string& w) {
  if (v.kind != JsonValue::Number) throw std::runtime_error("JSON key " + w + " is not a number");
  return v.num;
}
template <>
inline int ConfigData::Convert<int>(const JsonValue& v, const std::string& w) {
  if (v.kind != JsonValue::Number) throw std::runtime_error("JSON key " + w + " is not a number");
  return (int)v.num;
}
template <>
inline long long ConfigData::Convert<long long>(const JsonValue& v, const std::string& w) {
  if (v.kind != JsonValue::Number) throw std::runtime_error("JSON key " + w + " is not a number");
  return (long long)v.num;
}
template <>
inline std::string ConfigData::Convert<std::string>(const JsonValue& v, const std::string& w) {
  if (v.kind != JsonValue::String) throw std::runtime_error("JSON key " + w + " is not a string");
  return v.str;
}
template <>
inline bool ConfigData::Convert<bool>(const JsonValue& v, const std::string& w) {
  if (v.kind != JsonValue::Bool) throw std::runtime_error("JSON key " + w + " is not a bool");
  return v.b;
}

}  // namespace rbx_host
