// cqg_evolve — runs one of the reference's workload scripts on the B200 engine and writes
// the reference's trajectory file (the role of CPPQEDscripts/<script> with --o), through the
// C++ host side of include/cqg_ensemble.hpp over the engine's C ABI.
//
//   cqg_evolve <script> [--name value ...] [--o <file>]
//
// script: PTLA_C++QED, PumpedLossyMode_C++QED, QbitMode_C++QED, Optomechanics, 1particle1mode,
// Ring, QbitChain; the parameters are the reference script's (parameters::Table syntax).
// Without --o the trajectory goes to standard output, as in the reference.
#include <fstream>
#include <iostream>

#include "cqg_ensemble.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: cqg_evolve <script> [--name value ...] [--o <file>]\n";
    return 2;
  }
  std::vector<std::string> args;
  std::string out;
  for (int i = 2; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--o" && i + 1 < argc) {
      out = argv[++i];
      continue;
    }
    args.push_back(a);
  }
  try {
    if (out.empty()) {
      cqg::evolve(argv[1], args, std::cout);
    } else {
      std::ofstream f(out);
      if (!f) {
        std::cerr << "cannot open " << out << "\n";
        return 1;
      }
      cqg::evolve(argv[1], args, f);
    }
  } catch (const cqg::Error& e) {
    std::cerr << "cqg_evolve: " << e.what() << " (code " << e.code << ")\n";
    return 1;
  } catch (const std::exception& e) {
    std::cerr << "cqg_evolve: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
