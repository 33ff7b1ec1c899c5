#include "pars.hpp"

namespace cqg {

void ParameterTable::parse(const std::vector<std::string>& args) {
  for (size_t i = 0; i < args.size(); ++i) {
    const std::string& a = args[i];
    if (a.size() < 3 || a[0] != '-' || a[1] != '-')
      throw std::invalid_argument("Syntax error in command line around \"" + a + "\"");
    std::string name = a.substr(2);
    const bool hasValue = i + 1 < args.size() && !(args[i + 1].size() >= 2 && args[i + 1][0] == '-' &&
                                                    args[i + 1][1] == '-');
    if (hasValue) {
      values_[name] = args[++i];
    } else if (name.rfind("no_", 0) == 0) {
      switches_[name.substr(3)] = false;
    } else {
      switches_[name] = true;
    }
  }
}

void ParameterTable::checkAllKnown() const {
  for (auto& kv : values_)
    if (!known_.count(kv.first)) throw std::invalid_argument("Problem in command line around \"" + kv.first + "\"");
  for (auto& kv : switches_)
    if (!known_.count(kv.first)) throw std::invalid_argument("Problem in command line around \"" + kv.first + "\"");
}

}  // namespace cqg
