// Oracle test infrastructure: a project-written stand-in for the Cubism
// ArgumentParser, the command-line / key=value parser that the reference's
// Simulation.cpp, Shape.cpp and Utils/FactoryFileLineParser.h include
// (Cubism is an empty git submodule in the reference tree, .gitmodules:1-3).
//
// Behaviour restated from how the reference uses it:
//  - keys are stored WITHOUT a leading '-', and looked up with or without it
//    (Shape.cpp:332-345 queries "-xvel"; FactoryFileLineParser.h:52 stores
//    "xvel"), so operator() strips one leading '-';
//  - Value::asDouble/asInt/asBool/asString return the default when the key is
//    absent; in strict mode (Simulation.cpp:72-75) a missing key aborts.
#pragma once
// The reference relies on Cubism's headers to pull in these standard headers
// (e.g. ObstacleBlock.h:129-136 uses std::ofstream without including it).
#include <array>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <iostream>

namespace cubism {

class Value
{
  std::string content;
  bool present = false;
 public:
  Value() = default;
  explicit Value(const std::string& c) : content(c), present(true) {}
  bool exists() const { return present; }
  double asDouble(double def = 0) {
    if (!present || content.empty()) { content = std::to_string(def); present = true; return def; }
    return std::atof(content.c_str());
  }
  int asInt(int def = 0) {
    if (!present || content.empty()) { content = std::to_string(def); present = true; return def; }
    return std::atoi(content.c_str());
  }
  bool asBool(bool def = false) {
    if (!present || content.empty()) { content = def ? "true" : "false"; present = true; return def; }
    if (content == "true" || content == "True" || content == "TRUE") return true;
    if (content == "false" || content == "False" || content == "FALSE") return false;
    return std::atoi(content.c_str()) != 0;
  }
  std::string asString(const std::string& def = "") {
    if (!present) { content = def; present = true; return def; }
    return content;
  }
};

class CommandlineParser
{
 protected:
  std::map<std::string, Value> mapArguments;
  bool bStrictMode = false;
  bool bVerbose = true;

  static std::string strip(std::string k) {
    if (!k.empty() && k[0] == '-') k.erase(0, 1);
    return k;
  }
 public:
  CommandlineParser(int argc, char** argv)
  {
    for (int i = 1; i < argc; i++) {
      if (argv[i][0] != '-') continue;
      std::string key = strip(argv[i]);
      std::string val;
      int j = i + 1;
      // a value is everything up to the next token that starts with '-'
      // followed by a non-digit (negative numbers are values)
      for (; j < argc; j++) {
        const char* a = argv[j];
        const bool isKey = a[0] == '-' && a[1] != 0 &&
          !(a[1] >= '0' && a[1] <= '9') && a[1] != '.';
        if (isKey) break;
        if (!val.empty()) val += " ";
        val += a;
      }
      mapArguments[key] = Value(val);
      i = j - 1;
    }
  }
  Value& operator()(const std::string& key)
  {
    const std::string k = strip(key);
    auto it = mapArguments.find(k);
    if (it == mapArguments.end()) {
      if (bStrictMode) {
        std::fprintf(stderr, "runtime argument -%s is required\n", k.c_str());
        std::abort();
      }
      return mapArguments[k];
    }
    return it->second;
  }
  bool check(const std::string& key) const {
    return mapArguments.find(strip(key)) != mapArguments.end();
  }
  void set_strict_mode() { bStrictMode = true; }
  void unset_strict_mode() { bStrictMode = false; }
  void mute() { bVerbose = false; }
  void loud() { bVerbose = true; }
  void print_args() {}
};

class ArgumentParser : public CommandlineParser
{
 public:
  ArgumentParser(int argc, char** argv, char cl = '#', char sp = ' ')
    : CommandlineParser(argc, argv) { (void)cl; (void)sp; }
};

} // namespace cubism
