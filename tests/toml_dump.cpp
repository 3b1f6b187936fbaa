// Prints a TOML file parsed by the shim's reader as JSON (test helper: the
// CPU tests compare it with Python's tomllib on the same file).
#include <cstdio>
#include <string>

#include "icarat_toml.hpp"

namespace toml = icarat_b200::toml;

static void dump(const toml::value &v)
{
  switch(v.kind())
  {
  case toml::value::INTEGER: std::printf("%lld", v.as_integer()); break;
  case toml::value::FLOAT:
  {
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v.as_floating());
    std::string t(b);
    if(t.find_first_of(".en") == std::string::npos)
      t += ".0";
    std::printf("%s", t.c_str());
    break;
  }
  case toml::value::BOOLEAN: std::printf(v.as_boolean() ? "true" : "false"); break;
  case toml::value::STRING:
  {
    std::string s;
    for(char c : v.as_string())
      s += (c == '"' || c == '\\') ? std::string("\\") + c : std::string(1, c);
    std::printf("\"%s\"", s.c_str());
    break;
  }
  case toml::value::ARRAY:
  {
    std::printf("[");
    bool first = true;
    for(const toml::value &e : v.as_array())
    {
      std::printf(first ? "" : ",");
      first = false;
      dump(e);
    }
    std::printf("]");
    break;
  }
  case toml::value::TABLE:
  {
    std::printf("{");
    bool first = true;
    for(const auto &kv : v.as_table())
    {
      std::printf(first ? "\"%s\":" : ",\"%s\":", kv.first.c_str());
      first = false;
      dump(kv.second);
    }
    std::printf("}");
    break;
  }
  default: std::printf("null");
  }
}

int main(int argc, char **argv)
{
  try
  {
    for(int i = 1; i < argc; i++)
    {
      dump(toml::parse(argv[i]));
      std::printf("\n");
    }
  }
  catch(const std::exception &e)
  {
    std::printf("ERROR %s\n", e.what());
    return 2;
  }
  return 0;
}
