#include "errors.hpp"

namespace cqg {

namespace {
thread_local std::string lastError;
}

void setLastError(const std::string& msg) { lastError = msg; }

int fail(int code, const std::string& msg) {
  lastError = msg;
  return code;
}

const char* lastErrorCStr() { return lastError.c_str(); }

}  // namespace cqg

extern "C" {

const char* cqg_last_error(void) { return cqg::lastErrorCStr(); }

int cqg_abi_version(void) { return CQG_ABI_VERSION; }

void cqg_mcwf_pars_default(cqg_mcwf_pars* p) {
  if (!p) return;
  *p = cqg_mcwf_pars{};
  p->eps_rel = 1e-6;
  p->eps_abs = 1e-12;
  p->dp_limit = 0.01;
  p->overshoot_tolerance = 10.;
  p->dt_init = 0.;
  p->seed = 1001;
  p->prng_stream = 1;
  p->rng = CQG_RNG_PCG64;
  p->noise = 1;
  p->precision = CQG_FP64;
  p->max_attempts = 0;
  p->autotune = 1;
  p->cta_threads = 0;
}

}  // extern "C"
