// icarat_toml.hpp -- the TOML subset ICARAT's input files use, without toml11.
//
// ICARAT reads its `.toml` inputs with toml11 (`toml::parse`, `toml::find<T>`,
// `toml::get<T>`).  The structured-box apps only need: `[table]` headers,
// `key = value` lines, integers, floats, booleans, basic strings, and arrays
// (nested, possibly spread over several lines, trailing commas allowed), with
// `#` comments.  This header parses exactly that and offers the same call
// shapes (find with one or two keys, conversion to int / double / bool /
// std::string / std::vector / std::array), so the shim's mesh, material and
// boundary-condition readers take the same keys ICARAT's do:
//   [mesh]                dimension, division, length, type
//     (src/io/mesh_icarat.hpp:69-128)
//   [material]            type, designs_0, penalty, young, poisson, state
//     (src/problem/elasticity.cpp:19-32)
//   [boundary_condition]  dirichlet = [[flag6], [val6], [[x0,x1],[y0,y1],[z0,z1]]] rows,
//                         neumann   = [[val3], [[x0,x1],[y0,y1],[z0,z1]]] rows
//     (src/io/boundary_condition_icarat.hpp:68-127, 253-291)
// Anything outside the subset (inline tables, dates, literal or multi-line
// strings, dotted keys) raises toml::syntax_error naming the line.
#pragma once
#include <array>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace icarat_b200
{
namespace toml
{

struct syntax_error : std::runtime_error
{
  using std::runtime_error::runtime_error;
};
struct type_error : std::runtime_error
{
  using std::runtime_error::runtime_error;
};

class value;
using array = std::vector<value>;
using table = std::map<std::string, value>;

class value
{
public:
  enum kind_t
  {
    EMPTY,
    INTEGER,
    FLOAT,
    BOOLEAN,
    STRING,
    ARRAY,
    TABLE
  };
  value() = default;
  static value integer(long long v)
  {
    value r;
    r.k_ = INTEGER;
    r.i_ = v;
    return r;
  }
  static value floating(double v)
  {
    value r;
    r.k_ = FLOAT;
    r.f_ = v;
    return r;
  }
  static value boolean(bool v)
  {
    value r;
    r.k_ = BOOLEAN;
    r.b_ = v;
    return r;
  }
  static value string(std::string v)
  {
    value r;
    r.k_ = STRING;
    r.s_ = std::move(v);
    return r;
  }
  static value make_array() { value r; r.k_ = ARRAY; return r; }
  static value make_table() { value r; r.k_ = TABLE; return r; }

  kind_t kind() const { return k_; }
  bool is_table() const { return k_ == TABLE; }
  bool is_array() const { return k_ == ARRAY; }

  long long as_integer() const
  {
    if(k_ != INTEGER)
      throw type_error("toml: value is not an integer");
    return i_;
  }
  /// integers convert to floating point (toml11 does the same for double)
  double as_floating() const
  {
    if(k_ == FLOAT)
      return f_;
    if(k_ == INTEGER)
      return double(i_);
    throw type_error("toml: value is not a number");
  }
  bool as_boolean() const
  {
    if(k_ != BOOLEAN)
      throw type_error("toml: value is not a boolean");
    return b_;
  }
  const std::string &as_string() const
  {
    if(k_ != STRING)
      throw type_error("toml: value is not a string");
    return s_;
  }
  const array &as_array() const
  {
    if(k_ != ARRAY)
      throw type_error("toml: value is not an array");
    return a_;
  }
  array &as_array()
  {
    if(k_ != ARRAY)
      throw type_error("toml: value is not an array");
    return a_;
  }
  const table &as_table() const
  {
    if(k_ != TABLE)
      throw type_error("toml: value is not a table");
    return t_;
  }
  table &as_table()
  {
    if(k_ != TABLE)
      throw type_error("toml: value is not a table");
    return t_;
  }
  bool contains(const std::string &key) const { return k_ == TABLE && t_.count(key) > 0; }
  const value &at(const std::string &key) const
  {
    const table &t = as_table();
    auto it = t.find(key);
    if(it == t.end())
      throw std::out_of_range("toml: key \"" + key + "\" not found");
    return it->second;
  }

private:
  kind_t k_ = EMPTY;
  long long i_ = 0;
  double f_ = 0.0;
  bool b_ = false;
  std::string s_;
  array a_;
  table t_;
};

// ---- conversions (toml::get<T>) -------------------------------------------
namespace detail
{
template <class T> struct conv;
template <> struct conv<int>
{
  static int get(const value &v) { return int(v.as_integer()); }
};
template <> struct conv<long long>
{
  static long long get(const value &v) { return v.as_integer(); }
};
template <> struct conv<double>
{
  static double get(const value &v) { return v.as_floating(); }
};
template <> struct conv<bool>
{
  static bool get(const value &v) { return v.as_boolean(); }
};
template <> struct conv<std::string>
{
  static std::string get(const value &v) { return v.as_string(); }
};
template <> struct conv<value>
{
  static value get(const value &v) { return v; }
};
template <> struct conv<array>
{
  static array get(const value &v) { return v.as_array(); }
};
template <class T> struct conv<std::vector<T>>
{
  static std::vector<T> get(const value &v)
  {
    std::vector<T> r;
    for(const value &e : v.as_array())
      r.push_back(conv<T>::get(e));
    return r;
  }
};
template <class T, std::size_t N> struct conv<std::array<T, N>>
{
  static std::array<T, N> get(const value &v)
  {
    const array &a = v.as_array();
    if(a.size() != N)
      throw type_error("toml: array has " + std::to_string(a.size()) + " entries, expected " +
                       std::to_string(N));
    std::array<T, N> r;
    for(std::size_t i = 0; i < N; i++)
      r[i] = conv<T>::get(a[i]);
    return r;
  }
};
} // namespace detail

template <class T> T get(const value &v) { return detail::conv<T>::get(v); }

inline const value &find(const value &v, const std::string &key) { return v.at(key); }
template <class T> T find(const value &v, const std::string &key) { return get<T>(v.at(key)); }
template <class T> T find(const value &v, const std::string &k1, const std::string &k2)
{
  return get<T>(v.at(k1).at(k2));
}

// ---- parser -----------------------------------------------------------------
namespace detail
{
class Parser
{
public:
  Parser(std::string text, std::string name) : s_(std::move(text)), name_(std::move(name)) {}

  value run()
  {
    value root = value::make_table();
    value *cur = &root;
    for(;;)
    {
      skipBlank(true);
      if(pos_ >= s_.size())
        break;
      char c = s_[pos_];
      if(c == '[')
      {
        pos_++;
        if(peek() == '[')
          fail("arrays of tables are outside the supported subset");
        skipSpaces();
        std::string key = bareKey();
        skipSpaces();
        expect(']');
        table &t = root.as_table();
        if(t.count(key))
          fail("table [" + key + "] defined twice");
        t[key] = value::make_table();
        cur = &t[key];
        endOfLine();
        continue;
      }
      std::string key = bareKey();
      skipSpaces();
      expect('=');
      skipSpaces();
      value v = parseValue();
      table &t = cur->as_table();
      if(t.count(key))
        fail("key \"" + key + "\" defined twice");
      t[key] = std::move(v);
      endOfLine();
    }
    return root;
  }

private:
  std::string s_, name_;
  std::size_t pos_ = 0;

  [[noreturn]] void fail(const std::string &what) const
  {
    int line = 1;
    for(std::size_t i = 0; i < pos_ && i < s_.size(); i++)
      line += s_[i] == '\n';
    throw syntax_error("toml: " + name_ + ":" + std::to_string(line) + ": " + what);
  }
  char peek() const { return pos_ < s_.size() ? s_[pos_] : '\0'; }
  void expect(char c)
  {
    if(peek() != c)
      fail(std::string("expected '") + c + "'");
    pos_++;
  }
  void skipSpaces()
  {
    while(pos_ < s_.size() && (s_[pos_] == ' ' || s_[pos_] == '\t'))
      pos_++;
  }
  void skipComment()
  {
    if(peek() == '#')
      while(pos_ < s_.size() && s_[pos_] != '\n')
        pos_++;
  }
  /// spaces, comments and (when newlines) line breaks
  void skipBlank(bool newlines)
  {
    for(;;)
    {
      skipSpaces();
      skipComment();
      if(newlines && pos_ < s_.size() && (s_[pos_] == '\n' || s_[pos_] == '\r'))
      {
        pos_++;
        continue;
      }
      return;
    }
  }
  void endOfLine()
  {
    skipSpaces();
    skipComment();
    if(pos_ < s_.size() && s_[pos_] == '\r')
      pos_++;
    if(pos_ < s_.size() && s_[pos_] != '\n')
      fail("unexpected text after the value");
  }
  std::string bareKey()
  {
    if(peek() == '"')
      return quoted();
    std::size_t b = pos_;
    while(pos_ < s_.size() && (std::isalnum((unsigned char)s_[pos_]) || s_[pos_] == '_' ||
                               s_[pos_] == '-'))
      pos_++;
    if(b == pos_)
      fail("expected a key");
    if(peek() == '.')
      fail("dotted keys are outside the supported subset");
    return s_.substr(b, pos_ - b);
  }
  std::string quoted()
  {
    expect('"');
    std::string r;
    while(pos_ < s_.size() && s_[pos_] != '"')
    {
      char c = s_[pos_++];
      if(c == '\n')
        fail("newline inside a string");
      if(c == '\\')
      {
        char e = peek();
        pos_++;
        switch(e)
        {
        case 'n': r += '\n'; break;
        case 't': r += '\t'; break;
        case '\\': r += '\\'; break;
        case '"': r += '"'; break;
        default: fail("unsupported escape in a string");
        }
      }
      else
        r += c;
    }
    expect('"');
    return r;
  }
  value parseValue()
  {
    char c = peek();
    if(c == '"')
      return value::string(quoted());
    if(c == '[')
    {
      pos_++;
      value a = value::make_array();
      skipBlank(true);
      while(peek() != ']')
      {
        a.as_array().push_back(parseValue());
        skipBlank(true);
        if(peek() == ',')
        {
          pos_++;
          skipBlank(true);
        }
        else if(peek() != ']')
          fail("expected ',' or ']' in an array");
      }
      pos_++;
      return a;
    }
    if(c == '{')
      fail("inline tables are outside the supported subset");
    if(s_.compare(pos_, 4, "true") == 0)
    {
      pos_ += 4;
      return value::boolean(true);
    }
    if(s_.compare(pos_, 5, "false") == 0)
    {
      pos_ += 5;
      return value::boolean(false);
    }
    std::size_t b = pos_;
    while(pos_ < s_.size() && (std::isdigit((unsigned char)s_[pos_]) || s_[pos_] == '+' ||
                               s_[pos_] == '-' || s_[pos_] == '.' || s_[pos_] == 'e' ||
                               s_[pos_] == 'E' || s_[pos_] == '_'))
      pos_++;
    std::string tok;
    for(std::size_t i = b; i < pos_; i++)
      if(s_[i] != '_')
        tok += s_[i];
    if(tok.empty())
      fail("expected a value");
    bool isFloat = tok.find_first_of(".eE") != std::string::npos;
    char *end = nullptr;
    if(isFloat)
    {
      double v = std::strtod(tok.c_str(), &end);
      if(*end)
        fail("bad number \"" + tok + "\"");
      return value::floating(v);
    }
    long long v = std::strtoll(tok.c_str(), &end, 10);
    if(*end)
      fail("bad integer \"" + tok + "\"");
    return value::integer(v);
  }
};
} // namespace detail

inline value parse_string(const std::string &text, const std::string &name = "<string>")
{
  return detail::Parser(text, name).run();
}

/// toml::parse(path) as ICARAT's apps call it (opt_mma_Helmholtz.cpp:25)
inline value parse(const std::string &path)
{
  std::ifstream in(path);
  if(!in)
    throw std::runtime_error("toml: cannot open " + path);
  std::stringstream ss;
  ss << in.rdbuf();
  return parse_string(ss.str(), path);
}

} // namespace toml
} // namespace icarat_b200
