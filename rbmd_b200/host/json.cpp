// json.cpp -- recursive-descent reader for the RBMD input dialect (see json.hpp).
#include "json.hpp"

#include <cstdlib>
#include <fstream>
#include <sstream>

namespace rbmd_host {

const Json* Json::find(const std::string& key) const {
  if (type != Object) return nullptr;
  for (const auto& kv : obj)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

double Json::number(const std::string& key, double dflt) const {
  const Json* v = find(key);
  if (!v) return dflt;
  if (v->type == Number) return v->num;
  if (v->type == Bool) return v->b ? 1.0 : 0.0;
  throw std::runtime_error("json: key \"" + key + "\" is not a number");
}

std::string Json::string(const std::string& key, const std::string& dflt) const {
  const Json* v = find(key);
  if (!v) return dflt;
  if (v->type == String) return v->str;
  throw std::runtime_error("json: key \"" + key + "\" is not a string");
}

bool Json::boolean(const std::string& key, bool dflt) const {
  const Json* v = find(key);
  if (!v) return dflt;
  if (v->type == Bool) return v->b;
  if (v->type == Number) return v->num != 0.0;
  if (v->type == String) return v->str == "true";
  throw std::runtime_error("json: key \"" + key + "\" is not a boolean");
}

std::vector<double> Json::numbers(const std::string& key) const {
  std::vector<double> out;
  const Json* v = find(key);
  if (!v) return out;
  if (v->type == Number) return {v->num};
  if (v->type != Array) throw std::runtime_error("json: key \"" + key + "\" is not an array");
  for (const auto& e : v->arr) {
    if (e.type != Number) throw std::runtime_error("json: key \"" + key + "\" holds a non-number");
    out.push_back(e.num);
  }
  return out;
}

namespace {

struct Reader {
  const std::string& t;
  size_t p = 0;

  [[noreturn]] void fail(const std::string& what) const {
    int line = 1, col = 1;
    for (size_t k = 0; k < p && k < t.size(); ++k) {
      if (t[k] == '\n') {
        ++line;
        col = 1;
      } else {
        ++col;
      }
    }
    throw std::runtime_error("json: " + what + " at line " + std::to_string(line) + " column " +
                             std::to_string(col));
  }

  void skip() {  // white space and comments
    for (;;) {
      while (p < t.size() && (t[p] == ' ' || t[p] == '\t' || t[p] == '\n' || t[p] == '\r')) ++p;
      if (p + 1 < t.size() && t[p] == '/' && t[p + 1] == '/') {
        while (p < t.size() && t[p] != '\n') ++p;
      } else if (p + 1 < t.size() && t[p] == '/' && t[p + 1] == '*') {
        const size_t e = t.find("*/", p + 2);
        if (e == std::string::npos) fail("unterminated comment");
        p = e + 2;
      } else {
        return;
      }
    }
  }

  bool eat(char c) {
    skip();
    if (p < t.size() && t[p] == c) {
      ++p;
      return true;
    }
    return false;
  }

  std::string str() {
    if (!eat('"')) fail("expected a string");
    std::string out;
    while (p < t.size() && t[p] != '"') {
      char c = t[p++];
      if (c == '\\') {
        if (p >= t.size()) fail("bad escape");
        const char e = t[p++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {  // keep the code point as UTF-8
            if (p + 4 > t.size()) fail("bad \\u escape");
            const unsigned cp = (unsigned)std::strtoul(t.substr(p, 4).c_str(), nullptr, 16);
            p += 4;
            if (cp < 0x80) {
              out += (char)cp;
            } else if (cp < 0x800) {
              out += (char)(0xc0 | (cp >> 6));
              out += (char)(0x80 | (cp & 0x3f));
            } else {
              out += (char)(0xe0 | (cp >> 12));
              out += (char)(0x80 | ((cp >> 6) & 0x3f));
              out += (char)(0x80 | (cp & 0x3f));
            }
            break;
          }
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (p >= t.size()) fail("unterminated string");
    ++p;
    return out;
  }

  Json value() {
    skip();
    if (p >= t.size()) fail("unexpected end of input");
    Json v;
    const char c = t[p];
    if (c == '{') {
      ++p;
      v.type = Json::Object;
      for (;;) {
        if (eat('}')) break;
        std::string k = str();
        if (!eat(':')) fail("expected ':'");
        v.obj.emplace_back(std::move(k), value());
        if (eat(',')) continue;  // a trailing comma is accepted by the '}' test above
        if (eat('}')) break;
        fail("expected ',' or '}'");
      }
    } else if (c == '[') {
      ++p;
      v.type = Json::Array;
      for (;;) {
        if (eat(']')) break;
        v.arr.push_back(value());
        if (eat(',')) continue;
        if (eat(']')) break;
        fail("expected ',' or ']'");
      }
    } else if (c == '"') {
      v.type = Json::String;
      v.str = str();
    } else if (t.compare(p, 4, "true") == 0) {
      p += 4;
      v.type = Json::Bool;
      v.b = true;
    } else if (t.compare(p, 5, "false") == 0) {
      p += 5;
      v.type = Json::Bool;
    } else if (t.compare(p, 4, "null") == 0) {
      p += 4;
    } else {
      const char* s = t.c_str() + p;
      char* e = nullptr;
      v.num = std::strtod(s, &e);
      if (e == s) fail("unexpected character");
      v.type = Json::Number;
      p += (size_t)(e - s);
    }
    return v;
  }
};

}  // namespace

Json parse_json(const std::string& text) {
  std::string t = text;
  if (t.size() >= 3 && (unsigned char)t[0] == 0xef && (unsigned char)t[1] == 0xbb && (unsigned char)t[2] == 0xbf)
    t.erase(0, 3);
  Reader r{t};
  Json v = r.value();
  r.skip();
  if (r.p != t.size()) r.fail("trailing characters");
  return v;
}

Json parse_json_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parse_json(ss.str());
}

}  // namespace rbmd_host
