// Project-written stand-in for the part of Boost.PropertyTree that the
// reference's INI reader uses (file_access.cpp:36-75): a tree of string
// values addressed by "section.key" paths, get<T>() with Boost's
// translation rules, and the ptree_error exception family.  It lets the
// reference's own file_access.cpp compile unmodified where Boost is absent.
#ifndef MHD2D_B200_SHIM_PTREE_HPP
#define MHD2D_B200_SHIM_PTREE_HPP

#include <cstdio>
#include <ios>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace boost {
namespace property_tree {

class ptree_error : public std::runtime_error {
 public:
  explicit ptree_error(const std::string& what) : std::runtime_error(what) {}
};
class ptree_bad_data : public ptree_error {
 public:
  explicit ptree_bad_data(const std::string& what) : ptree_error(what) {}
};
class ptree_bad_path : public ptree_error {
 public:
  explicit ptree_bad_path(const std::string& what) : ptree_error(what) {}
};

namespace detail {
// Boost's stream translation: the whole value (up to trailing white space)
// must be consumed; bool also accepts "true" / "false".  White space is
// skipped only before the end of the value: an extraction on a stream
// already at its end would fail.
template <class T>
inline bool translate(const std::string& data, T& out) {
  std::istringstream is(data);
  T v;
  is >> v;
  if (!is.fail() && !is.eof()) is >> std::ws;
  if (is.fail() || is.bad() || is.get() != std::char_traits<char>::eof()) return false;
  out = v;
  return true;
}
inline bool translate(const std::string& data, bool& out) {
  std::istringstream is(data);
  bool v = false;
  is >> v;
  if (is.fail()) {
    is.clear();
    is.setf(std::ios_base::boolalpha);
    is >> v;
  }
  if (!is.fail() && !is.eof()) is >> std::ws;
  if (is.fail() || is.bad() || is.get() != std::char_traits<char>::eof()) return false;
  out = v;
  return true;
}
inline bool translate(const std::string& data, std::string& out) {
  out = data;
  return true;
}
}  // namespace detail

// A node: its own value and its children in insertion order.
class ptree {
 public:
  ptree() {}
  explicit ptree(const std::string& data) : data_(data) {}

  const std::string& data() const { return data_; }

  // Child by key (one level), nullptr if absent.
  const ptree* find_child(const std::string& key) const {
    for (const auto& kv : children_)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  ptree& push_back(const std::string& key, const ptree& child) {
    children_.emplace_back(key, child);
    return children_.back().second;
  }
  size_t size() const { return children_.size(); }

  // Node at a '.'-separated path, nullptr if absent.
  const ptree* find_path(const std::string& path) const {
    const ptree* node = this;
    size_t start = 0;
    for (;;) {
      const size_t dot = path.find('.', start);
      const std::string key = path.substr(start, dot == std::string::npos ? std::string::npos
                                                                          : dot - start);
      node = node->find_child(key);
      if (!node || dot == std::string::npos) return node;
      start = dot + 1;
    }
  }

  template <class T>
  T get(const std::string& path) const {
    const ptree* node = find_path(path);
    if (!node) throw ptree_bad_path("No such node (" + path + ")");
    T value{};
    if (!detail::translate(node->data_, value))
      throw ptree_bad_data("conversion of data to type failed (" + path + ")");
    return value;
  }

 private:
  std::string data_;
  std::vector<std::pair<std::string, ptree>> children_;
};

}  // namespace property_tree
}  // namespace boost

#endif
