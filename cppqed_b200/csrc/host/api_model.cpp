// extern "C" surface of the host model builder (include/cqg_model.h).
#include <cstring>
#include <exception>
#include <string>

#include "cqg_model.h"
#include "errors.hpp"
#include "model.hpp"

struct cqg_model {
  std::unique_ptr<cqg::Model> m;
};

using cqg::guarded;

extern "C" {

int cqg_model_create(const char* script, int32_t argc, const char* const* argv, cqg_model** out) {
  return guarded([&] {
    if (!script || !out || argc < 0) return cqg::fail(CQG_E_INVALID, "cqg_model_create: null argument");
    std::vector<std::string> args;
    for (int i = 0; i < argc; ++i) args.emplace_back(argv[i]);
    auto h = new cqg_model{cqg::makeModel(script, args)};
    *out = h;
    return CQG_OK;
  });
}

int cqg_model_desc(const cqg_model* m, const cqg_system_desc** out) {
  if (!m || !out) return cqg::fail(CQG_E_INVALID, "null argument");
  *out = &m->m->sys->desc();
  return CQG_OK;
}

int cqg_model_dimension(const cqg_model* m, int64_t* d) {
  if (!m || !d) return cqg::fail(CQG_E_INVALID, "null argument");
  *d = int64_t(m->m->sys->totalDimension());
  return CQG_OK;
}

int cqg_model_initial_state(const cqg_model* m, cqg_complex* psi) {
  if (!m || !psi) return cqg::fail(CQG_E_INVALID, "null argument");
  for (size_t i = 0; i < m->m->psi0.size(); ++i) psi[i] = {m->m->psi0[i].real(), m->m->psi0[i].imag()};
  return CQG_OK;
}

int cqg_model_run_pars(const cqg_model* m, cqg_run_pars* out) {
  if (!m || !out) return cqg::fail(CQG_E_INVALID, "null argument");
  const auto& pe = m->m->pe;
  *out = cqg_run_pars{};
  out->T = pe.T;
  out->Dt = pe.Dt;
  out->dc = pe.dc;
  out->NDt = pe.NDt;
  out->sdf = int32_t(pe.sdf);
  out->n_traj = int64_t(pe.nTraj);
  out->evol = pe.evol == "single" ? CQG_EVOL_SINGLE : pe.evol == "ensemble" ? CQG_EVOL_ENSEMBLE : CQG_EVOL_MASTER;
  out->log_level = pe.logLevel;
  cqg_mcwf_pars_default(&out->mcwf);
  out->mcwf.eps_rel = pe.epsRel;
  out->mcwf.eps_abs = pe.epsAbs;
  out->mcwf.dp_limit = pe.dpLimit;
  out->mcwf.overshoot_tolerance = pe.overshootTolerance;
  out->mcwf.seed = pe.seed;
  out->mcwf.prng_stream = pe.prngStream;
  out->mcwf.noise = pe.noise ? 1 : 0;
  out->mcwf.rng = pe.rng == "philox" ? CQG_RNG_PHILOX : CQG_RNG_PCG64;
  out->mcwf.precision = pe.prec == "fp32" ? CQG_FP32 : CQG_FP64;
  return CQG_OK;
}

int cqg_model_n_avr(const cqg_model* m, int32_t* n) {
  if (!m || !n) return cqg::fail(CQG_E_INVALID, "null argument");
  *n = m->m->sys->nAvr();
  return CQG_OK;
}

int cqg_model_process(const cqg_model* m, double* averages) {
  if (!m || !averages) return cqg::fail(CQG_E_INVALID, "null argument");
  m->m->sys->process(averages);
  return CQG_OK;
}

int cqg_model_key(const cqg_model* m, char* buf, size_t cap) {
  if (!m || !buf || !cap) return cqg::fail(CQG_E_INVALID, "null argument");
  std::string s;
  for (auto& l : m->m->sys->avLabels()) s += l + "\n";
  std::strncpy(buf, s.c_str(), cap - 1);
  buf[cap - 1] = 0;
  return CQG_OK;
}

namespace {
int copyText(const std::string& s, char* buf, size_t cap, size_t* needed) {
  if (needed) *needed = s.size() + 1;
  if (!buf) return CQG_OK;
  if (!cap) return cqg::fail(CQG_E_INVALID, "zero capacity");
  std::strncpy(buf, s.c_str(), cap - 1);
  buf[cap - 1] = 0;
  return CQG_OK;
}
}  // namespace

int cqg_model_key_text(const cqg_model* m, int32_t first_column, char* buf, size_t cap, size_t* needed) {
  if (!m) return cqg::fail(CQG_E_INVALID, "null argument");
  return guarded([&] { return copyText(m->m->sys->keyText(first_column), buf, cap, needed); });
}

int cqg_model_parameters_text(const cqg_model* m, char* buf, size_t cap, size_t* needed) {
  if (!m) return cqg::fail(CQG_E_INVALID, "null argument");
  return guarded([&] { return copyText(m->m->sys->parametersText(), buf, cap, needed); });
}

int cqg_model_command_line(const cqg_model* m, char* buf, size_t cap, size_t* needed) {
  if (!m) return cqg::fail(CQG_E_INVALID, "null argument");
  return guarded([&] { return copyText(m->m->commandLine, buf, cap, needed); });
}

int cqg_model_destroy(cqg_model* m) {
  delete m;
  return CQG_OK;
}

}  // extern "C"
