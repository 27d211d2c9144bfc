// spk_config.hpp -- libconfig-format configuration files for spk_params_t.
//
// The reference reads its `spooky.cfg` with libconfig (hyperrealm/libconfig,
// fetched unpinned by its CMakeLists.txt:55-72) through the lookups of
// Parameters::Parameters (src/parameters/parameters.cu:59-505).  This is an
// independent reader of the documented libconfig grammar, enough for those
// files:
//   setting  = name ('=' | ':') value [';' | ',']
//   value    = scalar | '[' scalars ']' (array) | '(' values ')' (list)
//            | '{' settings '}' (group)
//   scalar   = true/false (any case) | integer (decimal or 0x hex, optional
//              L/LL suffix: 64-bit; too large for 32 bits: 64-bit)
//            | float (a '.' or an exponent) | "string" (escapes \\ \" \n \r
//              \t \f \xNN; adjacent strings concatenate)
//   comments # ..., // ..., /* ... */
// Lookups follow libconfig's typed getters with its default options (no
// automatic conversion): an integer setting does not satisfy a float lookup,
// a float does not satisfy an integer lookup, only true/false satisfy a bool
// lookup, and a 64-bit integer satisfies an int lookup when it fits.  A failed
// lookup leaves the reference's default in place, as the reference does.
// Paths are dot-separated names with [n] for array/list elements
// ("physics.boxsize.[0]" or "physics.boxsize[0]").
#pragma once
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace spkcfg {

enum Type { T_GROUP, T_ARRAY, T_LIST, T_INT, T_INT64, T_FLOAT, T_BOOL, T_STRING };

struct Setting {
    Type type = T_GROUP;
    std::string name;
    long long ival = 0;
    double fval = 0.0;
    bool bval = false;
    std::string sval;
    std::vector<Setting> items;   // group members, array / list elements
};

class Parser {
public:
    Parser(const std::string& text) : s_(text) {}
    bool parse(Setting& root, std::string& err) {
        root.type = T_GROUP;
        if (!settings(root, true)) { err = err_; return false; }
        return true;
    }

private:
    const std::string& s_;
    size_t i_ = 0;
    int line_ = 1;
    std::string err_;

    bool fail(const std::string& what) {
        if (err_.empty()) err_ = "line " + std::to_string(line_) + ": " + what;
        return false;
    }
    int peek() const { return i_ < s_.size() ? (unsigned char)s_[i_] : -1; }
    void adv() {
        if (i_ < s_.size() && s_[i_] == '\n') line_++;
        i_++;
    }
    void skip() {
        for (;;) {
            const int c = peek();
            if (c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\f' || c == '\v') { adv(); continue; }
            if (c == '#' || (c == '/' && i_ + 1 < s_.size() && s_[i_ + 1] == '/')) {
                while (peek() != -1 && peek() != '\n') adv();
                continue;
            }
            if (c == '/' && i_ + 1 < s_.size() && s_[i_ + 1] == '*') {
                adv(); adv();
                while (peek() != -1 && !(peek() == '*' && i_ + 1 < s_.size() && s_[i_ + 1] == '/')) adv();
                if (peek() == -1) return;
                adv(); adv();
                continue;
            }
            return;
        }
    }
    static bool name_start(int c) { return (c >= 'A' && c <= 'Z') || (c >= 'a' && c <= 'z') || c == '*'; }
    static bool name_char(int c) { return name_start(c) || (c >= '0' && c <= '9') || c == '-' || c == '_'; }

    // settings until '}' (or end of text at top level)
    bool settings(Setting& grp, bool top) {
        for (;;) {
            skip();
            const int c = peek();
            if (c == -1) return top ? true : fail("unterminated group");
            if (c == '}') return top ? fail("unexpected '}'") : true;
            if (c == '@') return fail("@include directives are not supported");
            if (!name_start(c)) return fail(std::string("expected a setting name, found '") + (char)c + "'");
            Setting st;
            while (name_char(peek())) { st.name.push_back((char)peek()); adv(); }
            skip();
            if (peek() != '=' && peek() != ':') return fail("expected '=' or ':' after " + st.name);
            adv();
            if (!value(st)) return false;
            skip();
            if (peek() == ';' || peek() == ',') adv();
            for (const Setting& o : grp.items)
                if (o.name == st.name) return fail("duplicate setting " + st.name);
            grp.items.push_back(std::move(st));
        }
    }

    bool value(Setting& v) {
        skip();
        const int c = peek();
        if (c == '{') {
            adv();
            v.type = T_GROUP;
            if (!settings(v, false)) return false;
            adv();   // '}'
            return true;
        }
        if (c == '[' || c == '(') {
            const char close = c == '[' ? ']' : ')';
            v.type = c == '[' ? T_ARRAY : T_LIST;
            adv();
            skip();
            if (peek() == close) { adv(); return true; }
            for (;;) {
                Setting e;
                if (!value(e)) return false;
                if (v.type == T_ARRAY) {
                    if (e.type == T_GROUP || e.type == T_ARRAY || e.type == T_LIST)
                        return fail("arrays hold scalars only (use a list)");
                    if (!v.items.empty() && v.items[0].type != e.type &&
                        !((v.items[0].type == T_INT || v.items[0].type == T_INT64) && (e.type == T_INT || e.type == T_INT64)))
                        return fail("array elements must share one type");
                }
                v.items.push_back(std::move(e));
                skip();
                if (peek() == ',') {
                    adv();
                    skip();
                    if (peek() == close) return fail(std::string("trailing ',' before '") + close + "'");
                    continue;
                }
                if (peek() == close) { adv(); return true; }
                return fail(std::string("expected ',' or '") + close + "'");
            }
        }
        if (c == '"') return string_value(v);
        return scalar(v);
    }

    bool string_value(Setting& v) {
        v.type = T_STRING;
        for (;;) {
            if (peek() != '"') break;
            adv();
            for (;;) {
                const int c = peek();
                if (c == -1 || c == '\n') return fail("unterminated string");
                adv();
                if (c == '"') break;
                if (c == '\\') {
                    const int e = peek();
                    adv();
                    switch (e) {
                        case '\\': v.sval.push_back('\\'); break;
                        case '"': v.sval.push_back('"'); break;
                        case 'n': v.sval.push_back('\n'); break;
                        case 'r': v.sval.push_back('\r'); break;
                        case 't': v.sval.push_back('\t'); break;
                        case 'f': v.sval.push_back('\f'); break;
                        case 'x': {
                            int h = 0;
                            for (int k = 0; k < 2; k++) {
                                const int d = peek();
                                int dv;
                                if (d >= '0' && d <= '9') dv = d - '0';
                                else if (d >= 'a' && d <= 'f') dv = d - 'a' + 10;
                                else if (d >= 'A' && d <= 'F') dv = d - 'A' + 10;
                                else return fail("bad \\x escape");
                                h = h * 16 + dv;
                                adv();
                            }
                            v.sval.push_back((char)h);
                            break;
                        }
                        default: return fail("unknown escape in string");
                    }
                } else {
                    v.sval.push_back((char)c);
                }
            }
            skip();   // adjacent strings concatenate
        }
        return true;
    }

    bool scalar(Setting& v) {
        std::string tok;
        while (peek() != -1) {
            const int c = peek();
            if ((c >= '0' && c <= '9') || (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '.' || c == '+' ||
                c == '-' || c == '_') {
                tok.push_back((char)c);
                adv();
            } else {
                break;
            }
        }
        if (tok.empty()) return fail("expected a value");
        std::string low;
        for (char ch : tok) low.push_back((char)((ch >= 'A' && ch <= 'Z') ? ch - 'A' + 'a' : ch));
        if (low == "true" || low == "false") {
            v.type = T_BOOL;
            v.bval = low == "true";
            return true;
        }
        // integer: [+-]digits | [+-]0x hex, optional L / LL
        std::string body = tok;
        bool force64 = false;
        if (body.size() >= 2 && (body.back() == 'L' || body.back() == 'l')) {
            body.pop_back();
            if (!body.empty() && (body.back() == 'L' || body.back() == 'l')) body.pop_back();
            force64 = true;
        }
        {
            size_t k = 0;
            if (k < body.size() && (body[k] == '+' || body[k] == '-')) k++;
            const bool hex = body.size() > k + 2 && body[k] == '0' && (body[k + 1] == 'x' || body[k + 1] == 'X');
            bool isint = k < body.size();
            for (size_t m = hex ? k + 2 : k; m < body.size() && isint; m++) {
                const char ch = body[m];
                isint = hex ? ((ch >= '0' && ch <= '9') || (ch >= 'a' && ch <= 'f') || (ch >= 'A' && ch <= 'F'))
                            : (ch >= '0' && ch <= '9');
            }
            if (isint && (!hex || body.size() > k + 2)) {
                errno = 0;
                char* end = nullptr;
                const long long x = strtoll(body.c_str(), &end, hex ? 16 : 10);
                if (errno != 0 || *end != '\0') return fail("integer out of range: " + tok);
                v.ival = x;
                v.type = (force64 || x < INT_MIN || x > INT_MAX) ? T_INT64 : T_INT;
                return true;
            }
        }
        if (force64) return fail("bad integer: " + tok);
        // float: needs a '.' or an exponent
        if (tok.find('.') == std::string::npos && low.find('e') == std::string::npos) return fail("bad value: " + tok);
        char* end = nullptr;
        const double d = strtod(tok.c_str(), &end);
        if (end == tok.c_str() || *end != '\0') return fail("bad value: " + tok);
        v.type = T_FLOAT;
        v.fval = d;
        return true;
    }
};

// Lookup by path ("a.b.[0]", "a.b[0]").
inline const Setting* lookup(const Setting& root, const std::string& path) {
    const Setting* cur = &root;
    size_t i = 0;
    while (i < path.size()) {
        if (path[i] == '.') { i++; continue; }
        if (path[i] == '[') {
            const size_t j = path.find(']', i);
            if (j == std::string::npos) return nullptr;
            const long idx = strtol(path.substr(i + 1, j - i - 1).c_str(), nullptr, 10);
            if (cur->type != T_ARRAY && cur->type != T_LIST) return nullptr;
            if (idx < 0 || (size_t)idx >= cur->items.size()) return nullptr;
            cur = &cur->items[(size_t)idx];
            i = j + 1;
            continue;
        }
        size_t j = i;
        while (j < path.size() && path[j] != '.' && path[j] != '[') j++;
        const std::string nm = path.substr(i, j - i);
        if (cur->type != T_GROUP) return nullptr;
        const Setting* nx = nullptr;
        for (const Setting& st : cur->items)
            if (st.name == nm) { nx = &st; break; }
        if (!nx) return nullptr;
        cur = nx;
        i = j;
    }
    return cur;
}

inline bool get_int(const Setting& r, const char* p, int* out) {
    const Setting* s = lookup(r, p);
    if (!s) return false;
    if (s->type == T_INT || (s->type == T_INT64 && s->ival >= INT_MIN && s->ival <= INT_MAX)) {
        *out = (int)s->ival;
        return true;
    }
    return false;
}
inline bool get_float(const Setting& r, const char* p, double* out) {
    const Setting* s = lookup(r, p);
    if (!s || s->type != T_FLOAT) return false;
    *out = s->fval;
    return true;
}
inline bool get_bool(const Setting& r, const char* p, int* out) {
    const Setting* s = lookup(r, p);
    if (!s || s->type != T_BOOL) return false;
    *out = s->bval ? 1 : 0;
    return true;
}
inline bool get_string(const Setting& r, const char* p, std::string* out) {
    const Setting* s = lookup(r, p);
    if (!s || s->type != T_STRING) return false;
    *out = s->sval;
    return true;
}

}  // namespace spkcfg
