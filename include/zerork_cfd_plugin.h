/*
 * zerork_cfd_plugin.h -- drop-in C ABI of the cfd_plugin reactor solver,
 * backed by the sm_100a batched integrator.
 *
 * Same entry points, enums and conventions as the reference's
 * applications/cfd_plugin/zerork_cfd_plugin.h:11-87 so existing CFD codes
 * relink unchanged:
 *  - opaque handle; INVALID_HANDLE on a null handle, INVALID_FILENAME /
 *    INVALID_POINTER on null arguments (zerork_cfd_plugin.cpp:51-52,182,192);
 *  - T, P and mass fractions are caller-owned and updated in place, mass
 *    fractions reactor-major with a stride of the species count;
 *  - aux field pointers are borrowed and must outlive zerork_reactor_solve;
 *  - FAILED_SOLVE if any reactor's integration failed (its state is left
 *    unchanged), as zerork_reactor_manager.cpp:1123-1125;
 *  - a handle is not thread-safe; use one handle per host thread.
 * Every reactor is integrated on the current CUDA device (no CPU fallback).
 */
#ifndef ZERORK_CFD_PLUGIN_H
#define ZERORK_CFD_PLUGIN_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef ZERORK_CFD_PLUGIN_EXPORTS
#define ZERORK_CFD_PLUGIN_EXPORTS __attribute__((visibility("default")))
#endif

/* zerork_cfd_plugin.h:11-19 */
typedef enum _zerork_field_t {
  ZERORK_FIELD_DPDT,
  ZERORK_FIELD_COST,
  ZERORK_FIELD_GPU,
  ZERORK_FIELD_Y_SRC,
  ZERORK_FIELD_E_SRC,
  ZERORK_FIELD_IGNITION_TIME,
  ZERORK_FIELD_TEMPERATURE_DELTA
} zerork_field_t;

/* zerork_cfd_plugin.h:21-32 */
typedef enum _zerork_status_t {
  ZERORK_STATUS_SUCCESS = 0,
  ZERORK_STATUS_INVALID_HANDLE,
  ZERORK_STATUS_INVALID_FILENAME,
  ZERORK_STATUS_INVALID_FIELD_NAME,
  ZERORK_STATUS_INVALID_POINTER,
  ZERORK_STATUS_FAILED_MECHANISM_PARSE,
  ZERORK_STATUS_FAILED_OPTIONS_PARSE,
  ZERORK_STATUS_FAILED_SOLVE,
  ZERORK_STATUS_OPTION_NOT_DEFINED,
  ZERORK_STATUS_UNKNOWN_ERROR = 99
} zerork_status_t;

typedef struct zerork_handle_impl *zerork_handle;

/* Replaces zerork_reactor_init (zerork_cfd_plugin.cpp:32-45); option
 * defaults as ZeroRKReactorManager's constructor
 * (zerork_reactor_manager.cpp:49-101).  Returns NULL on allocation failure. */
zerork_handle ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_init(void);

/* YAML "key: value" options file (zerork_reactor_manager.cpp:135-191; keys
 * relative_tolerance, absolute_tolerance, max_steps, max_dt, ... as the
 * reference's options file).  Only keys present in the file are changed. */
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_read_options_file(const char *options_filename,
                                                                           zerork_handle handle);

/* zerork_cfd_plugin.cpp:56-75 (options "mech_filename", "therm_filename"). */
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_set_mechanism_files(const char *mech_file,
                                                                             const char *therm_file,
                                                                             zerork_handle handle);

/* Parse the mechanism and upload tables (zerork_reactor_manager.cpp:193-241);
 * FAILED_MECHANISM_PARSE on a parse error.  Called lazily by solve. */
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_load_mechanism(zerork_handle handle);

/* zerork_cfd_plugin.h:44-46.  Stored; the GPU integrator does not call it
 * (the reference calls it only from its CPU serial path, solver_cvode.cpp:251). */
typedef int (*zerork_callback_fn)(int reactor_id, int steps, double time, double dt,
                                  const double *y, const double *dy, void *cb_fn_data);

/* Integrate n_reactors constant-volume reactors for dt (zerork_cfd_plugin.cpp:
 * 158-175 -> ZeroRKReactorManager::SolveReactors).  T [K], P [Pa] and mf
 * (reactor-major, nsp per reactor) are updated in place; ZERORK_FIELD_COST
 * receives the step count (negative on failure), ZERORK_FIELD_GPU the GPU
 * time share, ZERORK_FIELD_TEMPERATURE_DELTA the temperature rise. */
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_solve(const int n_cycle, const double time,
                                                               const double dt, const int n_reactors,
                                                               double *T, double *P, double *mf,
                                                               zerork_handle handle);

zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_set_aux_field_pointer(zerork_field_t ft,
                                                                               double *field_pointer,
                                                                               zerork_handle handle);

/* Option setters always succeed (any name is stored, optionable.cpp:61-75);
 * getters return OPTION_NOT_DEFINED for unknown names. */
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_set_int_option(const char *option_name_chr,
                                                                        int option_value,
                                                                        zerork_handle handle);
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_set_double_option(const char *option_name_chr,
                                                                           double option_value,
                                                                           zerork_handle handle);
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_set_string_option(const char *option_name_chr,
                                                                           const char *option_value,
                                                                           zerork_handle handle);
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_get_int_option(const char *option_name_chr,
                                                                        int *option_value,
                                                                        zerork_handle handle);
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_get_double_option(const char *option_name_chr,
                                                                           double *option_value,
                                                                           zerork_handle handle);
/* strncpy into *option_value, at most string_length bytes
 * (zerork_cfd_plugin.cpp:139-153). */
zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_get_string_option(const char *option_name_chr,
                                                                           char **option_value,
                                                                           int string_length,
                                                                           zerork_handle handle);

zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_set_callback_fn(zerork_callback_fn fn,
                                                                         void *cb_fn_data,
                                                                         zerork_handle handle);

zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_set_reactor_ids(int *reactor_ids,
                                                                         zerork_handle handle);

zerork_status_t ZERORK_CFD_PLUGIN_EXPORTS zerork_reactor_free(zerork_handle handle);

#ifdef __cplusplus
}
#endif
#endif
