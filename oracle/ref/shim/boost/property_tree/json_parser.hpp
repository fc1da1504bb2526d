// Test infrastructure: JSON reader/writer for the ptree stand-in (see
// ptree.hpp), covering what the reference's tbox::PropertyTree reads:
// objects, arrays (children with empty names), strings, numbers, true,
// false and null, all held as strings as Boost's JSON parser holds them.
// Comments are not JSON and are rejected, as Boost rejects them.
#ifndef GFREF_SHIM_BOOST_JSON_PARSER_HPP
#define GFREF_SHIM_BOOST_JSON_PARSER_HPP
#include <cctype>
#include <fstream>
#include <istream>
#include <iterator>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>

#include "boost/property_tree/ptree.hpp"

namespace boost {
namespace property_tree {

class json_parser_error : public std::runtime_error {
 public:
  explicit json_parser_error(const std::string &m) : std::runtime_error(m) {}
};

namespace json_detail {

struct Reader {
  const std::string &s;
  size_t i = 0;
  explicit Reader(const std::string &src) : s(src) {}

  [[noreturn]] void fail(const char *what) const {
    throw json_parser_error(std::string("JSON: ") + what + " at offset " + std::to_string(i));
  }
  void ws() {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
  }
  char peek() {
    ws();
    if (i >= s.size()) fail("unexpected end");
    return s[i];
  }
  void expect(char c) {
    if (peek() != c) fail("unexpected character");
    ++i;
  }
  std::string str() {
    expect('"');
    std::string out;
    while (true) {
      if (i >= s.size()) fail("unterminated string");
      char c = s[i++];
      if (c == '"') break;
      if (c == '\\') {
        if (i >= s.size()) fail("bad escape");
        char e = s[i++];
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
            if (i + 4 > s.size()) fail("bad \\u escape");
            unsigned v = std::stoul(s.substr(i, 4), nullptr, 16);
            i += 4;
            if (v < 0x80) out += static_cast<char>(v);
            else if (v < 0x800) {
              out += static_cast<char>(0xC0 | (v >> 6));
              out += static_cast<char>(0x80 | (v & 0x3F));
            } else {
              out += static_cast<char>(0xE0 | (v >> 12));
              out += static_cast<char>(0x80 | ((v >> 6) & 0x3F));
              out += static_cast<char>(0x80 | (v & 0x3F));
            }
            break;
          }
          default: fail("bad escape");
        }
      } else {
        out += c;
      }
    }
    return out;
  }
  void value(ptree &t) {
    char c = peek();
    if (c == '{') {
      ++i;
      if (peek() == '}') { ++i; return; }
      while (true) {
        std::string k = str();
        expect(':');
        ptree child;
        value(child);
        t.push_back(ptree::value_type(k, child));
        char d = peek();
        ++i;
        if (d == '}') return;
        if (d != ',') fail("expected , or }");
      }
    } else if (c == '[') {
      ++i;
      if (peek() == ']') { ++i; return; }
      while (true) {
        ptree child;
        value(child);
        t.push_back(ptree::value_type(std::string(), child));
        char d = peek();
        ++i;
        if (d == ']') return;
        if (d != ',') fail("expected , or ]");
      }
    } else if (c == '"') {
      t.data() = str();
    } else {
      size_t a = i;
      while (i < s.size() && (std::isalnum(static_cast<unsigned char>(s[i])) || s[i] == '-' ||
                              s[i] == '+' || s[i] == '.'))
        ++i;
      if (a == i) fail("unexpected character");
      std::string tok = s.substr(a, i - a);
      if (tok != "true" && tok != "false" && tok != "null" &&
          !(std::isdigit(static_cast<unsigned char>(tok[0])) || tok[0] == '-'))
        fail("bad literal");
      t.data() = tok;
    }
  }
};

inline void write(std::ostream &os, const ptree &t, int ind) {
  std::string pad(ind, ' ');
  if (t.empty()) {
    os << '"' << t.data() << '"';
    return;
  }
  bool arr = true;
  for (auto &kv : t)
    if (!kv.first.empty()) arr = false;
  os << (arr ? "[\n" : "{\n");
  bool first = true;
  for (auto &kv : t) {
    if (!first) os << ",\n";
    first = false;
    os << pad << "    ";
    if (!arr) os << '"' << kv.first << "\": ";
    write(os, kv.second, ind + 4);
  }
  os << '\n' << pad << (arr ? "]" : "}");
}

}  // namespace json_detail

inline void read_json(std::istream &is, ptree &pt) {
  std::string src((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
  json_detail::Reader r(src);
  ptree t;
  r.value(t);
  r.ws();
  if (r.i != src.size()) r.fail("trailing characters");
  pt.swap(t);
}

inline void read_json(const std::string &file, ptree &pt) {
  std::ifstream is(file);
  if (!is) throw json_parser_error("cannot open file " + file);
  read_json(is, pt);
}

inline void write_json(std::ostream &os, const ptree &pt) {
  json_detail::write(os, pt, 0);
  os << '\n';
}

inline void write_json(const std::string &file, const ptree &pt) {
  std::ofstream os(file);
  if (!os) throw json_parser_error("cannot open file " + file);
  write_json(os, pt);
}

}  // namespace property_tree
}  // namespace boost
#endif
