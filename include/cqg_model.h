/*
 * cqg_model.h — host-side model builder of the MCWF engine (C ABI).
 *
 * Builds a quantum system from one of the reference's workload scripts with its
 * command-line interface (`--name value`, parameters::Table, CPPQEDutils/Pars.h:111-217),
 * using the element library (Mode, Qbit, PumpedTwoLevelAtom, JaynesCummings,
 * CoupledModes) and the binary / composite tensor-product rules
 * (BinarySystem.cc:194-239, Composite.tcc:178-303).  The result is a
 * cqg_system_desc (cqg.h) plus the initial state and the run parameters of
 * evolution::Pars (Evolution_.h:34-46).  Needs no GPU.
 */
#ifndef CQG_MODEL_H_INCLUDED
#define CQG_MODEL_H_INCLUDED

#include "cqg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cqg_model cqg_model;

#define CQG_EVOL_SINGLE 0
#define CQG_EVOL_ENSEMBLE 1
#define CQG_EVOL_MASTER 2

/* trajectory::Pars + evolution::Pars (Trajectory.h:77-114, Evolution_.h:34-46) */
typedef struct cqg_run_pars {
  double T, Dt;
  int32_t dc;
  int64_t NDt;
  int32_t sdf;
  int64_t n_traj;
  int32_t evol;          /* CQG_EVOL_* */
  int32_t log_level;
  cqg_mcwf_pars mcwf;
} cqg_run_pars;

/* script: "PTLA_C++QED", "PumpedLossyMode_C++QED", "QbitMode_C++QED",
 * "Optomechanics", "QbitChain".  argv excludes the program name. */
int cqg_model_create(const char* script, int32_t argc, const char* const* argv, cqg_model** out);
int cqg_model_desc(const cqg_model* m, const cqg_system_desc** out);
int cqg_model_dimension(const cqg_model* m, int64_t* total_dim);
int cqg_model_initial_state(const cqg_model* m, cqg_complex* psi);
int cqg_model_run_pars(const cqg_model* m, cqg_run_pars* out);
int cqg_model_n_avr(const cqg_model* m, int32_t* n_avr);
/* Averaged::process_v on a row of n_avr linear averages (in place), e.g.
 * VAR(n) = <n^2> - <n>^2 (Mode.cc:198-201). */
int cqg_model_process(const cqg_model* m, double* averages);
/* Column labels ("Key to data"), '\n'-separated, NUL-terminated. */
int cqg_model_key(const cqg_model* m, char* buf, size_t cap);
/* Text for a reference-format trajectory file header (trajectory::run's introduction,
 * Trajectory.h:535-545): the system's part of "Key to data" with its columns numbered from
 * first_column (each averaging element's title, then " 3. rho00" lines), the system's
 * parameter block (element descriptions, dimensions, characteristics, decay channels), and
 * the command line the model was built from.  Lines end in '\n'.  buf == NULL only reports
 * the size needed (with the NUL) in *needed; otherwise at most cap - 1 characters are copied. */
int cqg_model_key_text(const cqg_model* m, int32_t first_column, char* buf, size_t cap, size_t* needed);
int cqg_model_parameters_text(const cqg_model* m, char* buf, size_t cap, size_t* needed);
int cqg_model_command_line(const cqg_model* m, char* buf, size_t cap, size_t* needed);
int cqg_model_destroy(cqg_model* m);

#ifdef __cplusplus
}
#endif

#endif /* CQG_MODEL_H_INCLUDED */
