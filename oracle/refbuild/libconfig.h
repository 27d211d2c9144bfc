/* libconfig.h -- the subset of libconfig's C API (hyperrealm/libconfig) that
 * the reference's Parameters::Parameters (src/parameters/parameters.cu:59-506)
 * calls, declared so that the reference's own sources compile unchanged in
 * the timing build of oracle/refbuild.  The implementation
 * (libconfig_shim.cpp) answers the calls with the project's own reader of
 * the libconfig grammar (spooky-git_b200/csrc/spk_config.hpp), with
 * libconfig's typed-lookup rules (no automatic int/float conversion).
 * TEST AND MEASUREMENT INFRASTRUCTURE: not part of the library. */
#ifndef SPK_REFBUILD_LIBCONFIG_H
#define SPK_REFBUILD_LIBCONFIG_H

#define CONFIG_TRUE  1
#define CONFIG_FALSE 0

typedef struct config_setting_t config_setting_t;   /* an opaque node of the parsed tree */

typedef struct config_t {
    void* impl;          /* parsed tree and last error (owned) */
    int error_line;
    const char* error_text;
} config_t;

#ifdef __cplusplus
extern "C" {
#endif
void config_init(config_t* config);
void config_destroy(config_t* config);
int config_read_file(config_t* config, const char* filename);
int config_error_line(const config_t* config);
const char* config_error_text(const config_t* config);
int config_lookup_int(const config_t* config, const char* path, int* value);
int config_lookup_bool(const config_t* config, const char* path, int* value);
int config_lookup_float(const config_t* config, const char* path, double* value);
int config_lookup_string(const config_t* config, const char* path, const char** value);
config_setting_t* config_lookup(const config_t* config, const char* path);
int config_setting_length(const config_setting_t* setting);
const char* config_setting_get_string_elem(const config_setting_t* setting, int index);
#ifdef __cplusplus
}
#endif
#endif
