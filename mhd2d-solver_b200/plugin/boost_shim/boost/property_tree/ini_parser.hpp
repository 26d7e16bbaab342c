// Project-written stand-in for boost::property_tree::read_ini with Boost's
// INI rules: lines are trimmed; empty lines and lines starting with ';' or
// '#' are comments; "[name]" opens a section; "key = value" (both trimmed,
// the value taken verbatim up to the line end) adds a key to the current
// section.  A missing file, an unmatched '[', a line without '=', an empty
// key and duplicate section or key names throw ini_parser_error.
#ifndef MHD2D_B200_SHIM_INI_PARSER_HPP
#define MHD2D_B200_SHIM_INI_PARSER_HPP

#include <fstream>
#include <string>

#include "ptree.hpp"

namespace boost {
namespace property_tree {

class file_parser_error : public ptree_error {
 public:
  file_parser_error(const std::string& msg, const std::string& file, unsigned long line)
      : ptree_error((file.empty() ? std::string("<unspecified file>") : file) +
                    (line ? "(" + std::to_string(line) + ")" : std::string()) + ": " + msg) {}
};

namespace ini_parser {

class ini_parser_error : public file_parser_error {
 public:
  ini_parser_error(const std::string& msg, const std::string& file, unsigned long line)
      : file_parser_error(msg, file, line) {}
};

namespace detail {
inline std::string trim(const std::string& s) {
  const char* ws = " \t\r\n\f\v";
  const size_t a = s.find_first_not_of(ws);
  if (a == std::string::npos) return std::string();
  const size_t b = s.find_last_not_of(ws);
  return s.substr(a, b - a + 1);
}
}  // namespace detail

inline void read_ini(std::istream& stream, ptree& pt, const std::string& file = std::string()) {
  ptree local;
  ptree* section = nullptr;
  std::string line;
  unsigned long line_no = 0;
  while (std::getline(stream, line)) {
    ++line_no;
    line = detail::trim(line);
    if (line.empty() || line[0] == ';' || line[0] == '#') continue;
    if (line[0] == '[') {
      const size_t end = line.find(']');
      if (end == std::string::npos) throw ini_parser_error("unmatched '['", file, line_no);
      const std::string key = detail::trim(line.substr(1, end - 1));
      if (local.find_child(key)) throw ini_parser_error("duplicate section name", file, line_no);
      section = &local.push_back(key, ptree());
    } else {
      ptree& container = section ? *section : local;
      const size_t eq = line.find('=');
      if (eq == std::string::npos)
        throw ini_parser_error("'=' character not found in line", file, line_no);
      if (eq == 0) throw ini_parser_error("key expected", file, line_no);
      const std::string key = detail::trim(line.substr(0, eq));
      const std::string data = detail::trim(line.substr(eq + 1));
      if (container.find_child(key)) throw ini_parser_error("duplicate key name", file, line_no);
      container.push_back(key, ptree(data));
    }
  }
  pt = local;
}

inline void read_ini(const std::string& filename, ptree& pt) {
  std::ifstream stream(filename.c_str());
  if (!stream) throw ini_parser_error("cannot open file", filename, 0);
  read_ini(stream, pt, filename);
}

}  // namespace ini_parser

using ini_parser::read_ini;

}  // namespace property_tree
}  // namespace boost

#endif
