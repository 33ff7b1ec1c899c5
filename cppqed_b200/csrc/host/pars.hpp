// Command-line parameter table with the names, defaults and switch semantics of
// parameters::Table (CPPQEDutils/Pars.h:111-217, Pars.cc:125-163):
//  - every parameter is `--name value` (a modifier suffix is appended to the name);
//  - booleans are switches: `--name` sets true, `--no_name` sets false;
//  - complex values are read by operator>> (`(re,im)` or `re`).
#pragma once

#include <complex>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace cqg {

class ParameterTable {
 public:
  // Registers a parameter with its default; returns the supplied value if there is one.
  template <typename T>
  T add(const std::string& name, const std::string& mod, const T& def) {
    const std::string key = name + mod;
    known_.insert(key);
    auto it = values_.find(key);
    if (it == values_.end()) return def;
    T v{};
    std::istringstream is(it->second);
    is >> v;
    if (is.fail()) throw std::invalid_argument("Parameter \"" + key + "\" supplied with incorrect syntax");
    return v;
  }
  bool addSwitch(const std::string& name, const std::string& mod, bool def) {
    const std::string key = name + mod;
    known_.insert(key);
    auto it = switches_.find(key);
    return it == switches_.end() ? def : it->second;
  }

  // Parses the arguments after the program name.  `--name value` pairs are kept as
  // text and typed when the element registers the parameter; a `--name` not followed
  // by a value is a switch, `--no_name` its negation.
  void parse(const std::vector<std::string>& args);

  // Throws std::invalid_argument naming the first supplied parameter nobody registered
  // (the reference aborts with "Problem in command line around ...").
  void checkAllKnown() const;

  const std::string& commandLine() const { return commandLine_; }
  void setCommandLine(const std::string& s) { commandLine_ = s; }

 private:
  std::map<std::string, std::string> values_;
  std::map<std::string, bool> switches_;
  std::string commandLine_;
  std::set<std::string> known_;
};

}  // namespace cqg
