// json.hpp -- the JSON dialect of RBMD input files: standard JSON plus a UTF-8 byte-order mark,
// // and /* */ comments and trailing commas, all of which the reference's bundled files use
// (jsoncpp with comments allowed, framework/JsonParser.h:73-77).  Objects keep their key order.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace rbmd_host {

struct Json {
  enum Type { Null, Bool, Number, String, Array, Object };
  Type type = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;

  bool is_object() const { return type == Object; }
  bool is_array() const { return type == Array; }
  bool is_number() const { return type == Number; }
  bool is_string() const { return type == String; }
  bool is_bool() const { return type == Bool; }

  // member lookup (nullptr when absent or when this is not an object)
  const Json* find(const std::string& key) const;
  bool has(const std::string& key) const { return find(key) != nullptr; }
  // typed accessors; throw std::runtime_error naming the key when present with the wrong type
  double number(const std::string& key, double dflt) const;
  std::string string(const std::string& key, const std::string& dflt) const;
  bool boolean(const std::string& key, bool dflt) const;
  std::vector<double> numbers(const std::string& key) const;  // [] when absent
};

// Parses text; throws std::runtime_error("json: <what> at line L column C").
Json parse_json(const std::string& text);
// Reads and parses a file; throws std::runtime_error on I/O or syntax errors.
Json parse_json_file(const std::string& path);

}  // namespace rbmd_host
