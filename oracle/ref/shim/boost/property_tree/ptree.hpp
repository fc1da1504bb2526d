// Test infrastructure: a small stand-in for the boost::property_tree::ptree
// subset that the reference's tbox::PropertyTree (src/tbox/property_tree.*)
// uses, so the reference's grid classes can be configured from JSON in the
// oracle/_ref build.  Semantics follow Boost's published behaviour:
//  * every node has a string value and an ordered list of (name, child);
//  * paths separate names with '.', and a lookup takes the first child of
//    that name;
//  * values convert by stream extraction that must consume the whole string
//    (trailing white space allowed); bool also accepts "true"/"false";
//  * JSON arrays are children with empty names, JSON scalars are strings.
#ifndef GFREF_SHIM_BOOST_PTREE_HPP
#define GFREF_SHIM_BOOST_PTREE_HPP
#include <cstddef>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace boost {

// Boost's own headers bring this declaration in with ptree; the reference's
// PropertyTree names it as a friend.
namespace serialization {
class access;
}

template <typename T>
class optional {
 public:
  optional() : ok_(false), v_() {}
  explicit optional(const T &v) : ok_(true), v_(v) {}
  bool is_initialized() const { return ok_; }
  bool has_value() const { return ok_; }
  explicit operator bool() const { return ok_; }
  bool operator!() const { return !ok_; }
  const T &get() const { return v_; }
  const T &operator*() const { return v_; }

 private:
  bool ok_;
  T v_;
};

namespace property_tree {

class ptree_bad_path : public std::runtime_error {
 public:
  explicit ptree_bad_path(const std::string &p) : std::runtime_error("No such node (" + p + ")") {}
};

class ptree_bad_data : public std::runtime_error {
 public:
  explicit ptree_bad_data(const std::string &d)
      : std::runtime_error("conversion of data to type failed (" + d + ")") {}
};

namespace detail {
template <typename T>
inline bool convert(const std::string &s, T &out) {
  std::istringstream is(s);
  is >> out;
  if (is.fail()) return false;
  is >> std::ws;
  return is.eof();
}
inline bool convert(const std::string &s, std::string &out) {
  out = s;
  return true;
}
inline bool convert(const std::string &s, bool &out) {
  if (s == "true") { out = true; return true; }
  if (s == "false") { out = false; return true; }
  int v = 0;
  if (!convert<int>(s, v) || (v != 0 && v != 1)) return false;
  out = v != 0;
  return true;
}
template <typename T>
inline std::string to_string(const T &v) {
  std::ostringstream os;
  os.precision(17);
  os << v;
  return os.str();
}
inline std::string to_string(const std::string &v) { return v; }
inline std::string to_string(const char *v) { return std::string(v); }
inline std::string to_string(bool v) { return v ? "true" : "false"; }
}  // namespace detail

class ptree {
 public:
  using key_type = std::string;
  using data_type = std::string;
  using value_type = std::pair<const std::string, ptree>;
  using size_type = std::size_t;

 private:
  // Children are held by pointer so that ptree can name itself in its pair.
  std::string data_;
  std::vector<value_type *> kids_;

  template <typename P>
  class iter {
   public:
    iter(P *const *p) : p_(p) {}
    value_type &operator*() const { return **p_; }
    value_type *operator->() const { return *p_; }
    iter &operator++() { ++p_; return *this; }
    bool operator!=(const iter &o) const { return p_ != o.p_; }
    bool operator==(const iter &o) const { return p_ == o.p_; }

   private:
    P *const *p_;
  };

 public:
  using iterator = iter<value_type>;
  using const_iterator = iter<value_type>;

  ptree() {}
  explicit ptree(const std::string &d) : data_(d) {}
  ptree(const ptree &o) : data_(o.data_) {
    for (auto *k : o.kids_) kids_.push_back(new value_type(k->first, k->second));
  }
  ptree &operator=(const ptree &o) {
    if (this != &o) {
      ptree tmp(o);
      swap(tmp);
    }
    return *this;
  }
  ~ptree() {
    for (auto *k : kids_) delete k;
  }
  void swap(ptree &o) {
    data_.swap(o.data_);
    kids_.swap(o.kids_);
  }

  size_type size() const { return kids_.size(); }
  bool empty() const { return kids_.empty(); }
  const_iterator begin() const { return const_iterator(kids_.data()); }
  const_iterator end() const { return const_iterator(kids_.data() + kids_.size()); }
  iterator begin() { return iterator(kids_.data()); }
  iterator end() { return iterator(kids_.data() + kids_.size()); }

  const std::string &data() const { return data_; }
  std::string &data() { return data_; }

  iterator push_back(const value_type &v) {
    kids_.push_back(new value_type(v.first, v.second));
    return iterator(kids_.data() + kids_.size() - 1);
  }

  size_type count(const std::string &name) const {
    size_type c = 0;
    for (auto *k : kids_)
      if (k->first == name) ++c;
    return c;
  }

  // Path lookup ('.'-separated names, first match per name).
  const ptree *find_path(const std::string &path) const {
    const ptree *t = this;
    if (path.empty()) return t;
    size_t a = 0;
    while (true) {
      size_t b = path.find('.', a);
      std::string name = path.substr(a, b == std::string::npos ? std::string::npos : b - a);
      const ptree *next = nullptr;
      for (auto *k : t->kids_)
        if (k->first == name) { next = &k->second; break; }
      if (!next) return nullptr;
      t = next;
      if (b == std::string::npos) return t;
      a = b + 1;
    }
  }

  const ptree &get_child(const std::string &path) const {
    const ptree *t = find_path(path);
    if (!t) throw ptree_bad_path(path);
    return *t;
  }
  ptree &get_child(const std::string &path) {
    return const_cast<ptree &>(static_cast<const ptree &>(*this).get_child(path));
  }

  template <typename T>
  T get_value() const {
    T v{};
    if (!detail::convert(data_, v)) throw ptree_bad_data(data_);
    return v;
  }
  template <typename T>
  optional<T> get_value_optional() const {
    T v{};
    if (!detail::convert(data_, v)) return optional<T>();
    return optional<T>(v);
  }
  template <typename T>
  T get(const std::string &path) const {
    return get_child(path).get_value<T>();
  }
  template <typename T>
  T get(const std::string &path, const T &dflt) const {
    const ptree *t = find_path(path);
    if (!t) return dflt;
    auto o = t->get_value_optional<T>();
    return o ? o.get() : dflt;
  }
  template <typename T>
  optional<T> get_optional(const std::string &path) const {
    const ptree *t = find_path(path);
    if (!t) return optional<T>();
    return t->get_value_optional<T>();
  }

  // put/put_child create missing path components and replace the first
  // existing child of each name.
  ptree &put_child(const std::string &path, const ptree &value) {
    ptree &t = walk_create(path);
    t = value;
    return t;
  }
  template <typename T>
  ptree &put(const std::string &path, const T &value) {
    ptree &t = walk_create(path);
    t.data_ = detail::to_string(value);
    return t;
  }

 private:
  ptree &walk_create(const std::string &path) {
    ptree *t = this;
    if (path.empty()) return *t;
    size_t a = 0;
    while (true) {
      size_t b = path.find('.', a);
      std::string name = path.substr(a, b == std::string::npos ? std::string::npos : b - a);
      ptree *next = nullptr;
      for (auto *k : t->kids_)
        if (k->first == name) { next = &k->second; break; }
      if (!next) {
        t->kids_.push_back(new value_type(name, ptree()));
        next = &t->kids_.back()->second;
      }
      t = next;
      if (b == std::string::npos) return *t;
      a = b + 1;
    }
  }
};

}  // namespace property_tree
}  // namespace boost
#endif
