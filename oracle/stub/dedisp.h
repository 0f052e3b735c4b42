/*
 * Stand-in declarations for the external dedisp library, which the
 * reference's headers include (include/utils/exceptions.hpp:8,
 * include/transforms/dedisperser.hpp:2) but which is not installed.  The
 * oracle build never dedisperses: every entry point returns an error.
 * TEST INFRASTRUCTURE ONLY.
 */
#pragma once
#include <cstddef>
typedef int dedisp_error;
typedef int dedisp_bool;
typedef float dedisp_float;
typedef unsigned char dedisp_byte;
typedef unsigned long dedisp_size;
typedef struct dedisp_plan_struct* dedisp_plan;
enum { DEDISP_NO_ERROR = 0, DEDISP_NOT_AVAILABLE = 1 };
static inline const char* dedisp_get_error_string(dedisp_error) { return "dedisp is not available in this build"; }
static inline dedisp_error dedisp_create_plan_multi(dedisp_plan*, dedisp_size, dedisp_float, dedisp_float, dedisp_float, unsigned) { return DEDISP_NOT_AVAILABLE; }
static inline void dedisp_destroy_plan(dedisp_plan) {}
static inline dedisp_error dedisp_set_dm_list(dedisp_plan, const dedisp_float*, dedisp_size) { return DEDISP_NOT_AVAILABLE; }
static inline dedisp_error dedisp_generate_dm_list(dedisp_plan, dedisp_float, dedisp_float, dedisp_float, dedisp_float) { return DEDISP_NOT_AVAILABLE; }
static inline dedisp_size dedisp_get_dm_count(dedisp_plan) { return 0; }
static inline const dedisp_float* dedisp_get_dm_list(dedisp_plan) { return 0; }
static inline dedisp_error dedisp_set_killmask(dedisp_plan, const dedisp_bool*) { return DEDISP_NOT_AVAILABLE; }
static inline dedisp_size dedisp_get_max_delay(dedisp_plan) { return 0; }
static inline dedisp_error dedisp_execute(dedisp_plan, dedisp_size, const dedisp_byte*, dedisp_size, dedisp_byte*, dedisp_size, unsigned) { return DEDISP_NOT_AVAILABLE; }
