// libconfig_shim.cpp -- libconfig's C lookups (the subset in libconfig.h)
// over the project's own libconfig-grammar reader, for the reference timing
// build.  A failed lookup returns CONFIG_FALSE and leaves the output alone,
// as libconfig does; strings stay valid until config_destroy.
#include "libconfig.h"

#include <fstream>
#include <sstream>
#include <string>

#include "spk_config.hpp"

namespace {
struct Impl {
    spkcfg::Setting root;
    std::string err;
};
Impl* impl(const config_t* c) { return static_cast<Impl*>(c->impl); }
}  // namespace

extern "C" void config_init(config_t* c) {
    c->impl = new Impl();
    c->error_line = 0;
    c->error_text = nullptr;
}

extern "C" void config_destroy(config_t* c) {
    delete impl(c);
    c->impl = nullptr;
}

extern "C" int config_read_file(config_t* c, const char* filename) {
    std::ifstream f(filename);
    Impl* d = impl(c);
    if (!f) {
        d->err = std::string("cannot open ") + filename;
        c->error_line = 0;
        c->error_text = d->err.c_str();
        return CONFIG_FALSE;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    spkcfg::Parser parser(text);
    std::string err;
    if (!parser.parse(d->root, err)) {
        d->err = err;
        // the reader's messages start "line N: "
        c->error_line = err.rfind("line ", 0) == 0 ? std::atoi(err.c_str() + 5) : 0;
        c->error_text = d->err.c_str();
        return CONFIG_FALSE;
    }
    return CONFIG_TRUE;
}

extern "C" int config_error_line(const config_t* c) { return c->error_line; }
extern "C" const char* config_error_text(const config_t* c) { return c->error_text ? c->error_text : ""; }

extern "C" int config_lookup_int(const config_t* c, const char* path, int* value) {
    return spkcfg::get_int(impl(c)->root, path, value) ? CONFIG_TRUE : CONFIG_FALSE;
}
extern "C" int config_lookup_bool(const config_t* c, const char* path, int* value) {
    return spkcfg::get_bool(impl(c)->root, path, value) ? CONFIG_TRUE : CONFIG_FALSE;
}
extern "C" int config_lookup_float(const config_t* c, const char* path, double* value) {
    return spkcfg::get_float(impl(c)->root, path, value) ? CONFIG_TRUE : CONFIG_FALSE;
}
extern "C" int config_lookup_string(const config_t* c, const char* path, const char** value) {
    const spkcfg::Setting* s = spkcfg::lookup(impl(c)->root, path);
    if (!s || s->type != spkcfg::T_STRING) return CONFIG_FALSE;
    *value = s->sval.c_str();
    return CONFIG_TRUE;
}
extern "C" config_setting_t* config_lookup(const config_t* c, const char* path) {
    const spkcfg::Setting* s = spkcfg::lookup(impl(c)->root, path);
    return reinterpret_cast<config_setting_t*>(const_cast<spkcfg::Setting*>(s));
}
extern "C" int config_setting_length(const config_setting_t* setting) {
    const spkcfg::Setting* s = reinterpret_cast<const spkcfg::Setting*>(setting);
    if (!s) return 0;
    if (s->type == spkcfg::T_GROUP || s->type == spkcfg::T_ARRAY || s->type == spkcfg::T_LIST)
        return (int)s->items.size();
    return 0;
}
extern "C" const char* config_setting_get_string_elem(const config_setting_t* setting, int index) {
    const spkcfg::Setting* s = reinterpret_cast<const spkcfg::Setting*>(setting);
    if (!s || (s->type != spkcfg::T_ARRAY && s->type != spkcfg::T_LIST)) return nullptr;
    if (index < 0 || (size_t)index >= s->items.size()) return nullptr;
    const spkcfg::Setting& e = s->items[(size_t)index];
    return e.type == spkcfg::T_STRING ? e.sval.c_str() : nullptr;
}
